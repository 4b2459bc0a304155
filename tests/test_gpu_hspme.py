"""GPU tests of the SPME with optiBasis's Hermite interpolation basis and its
adjoints (md_hspme_*, mdforce.optibasis.HermiteSPME), on the charged-fluid
system of the SPME-adjoint configuration (20736 +-1 charges, 30^3 box, mesh
64^3, beta 0.95) with a batch of 8 candidate bases of 32 coefficients (16
bins), the B-spline start of optiBasis/compute_basis.py:80-93 plus seeded
N(0, 0.1) perturbations, for orders 4 and 6:
  - with the basis of the order-4 cardinal B-spline (exactly representable by
    cubic Hermite pieces) the energy and forces are those of the reference
    B-spline SPME (md_spme, pinned to RE/src/EleRecBSpline.cpp built here);
  - the gradients of the energy and of the force-error functional with
    respect to the basis coefficients, the charges and the positions equal
    FP64 central differences (h = 1e-6; 1e-4 for the energy in q and r, whose
    rounding h = 1e-6 would amplify) to 1e-6 relative;
  - on a small system every output equals the numpy restatement
    (oracle/hspme.py) to 1e-11;
  - the torch.autograd.Functions hand those gradients back;
  - the measured force error of the B-spline basis is of the size of the
    optiBasis error estimate (optiBasis/IkError.py:123-136) of that basis."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

K = (64, 64, 64)
BETA = 0.95
NBIN = 16
TOL = 1e-6


@pytest.fixture(scope="module")
def fluid(mdf):
    import torch
    s = mdf.systems.charged_fluid()
    q = torch.tensor(s.charge, dtype=torch.float64, device="cuda")
    r = torch.tensor(s.pos, dtype=torch.float64, device="cuda")
    return s, q, r


@pytest.fixture(scope="module")
def fref(mdf, fluid):
    """Exact reciprocal Ewald forces (|m_d| <= 39, truncation below 1e-12)."""
    import torch
    s, _, _ = fluid
    sys = mdf.MDSystem(s.pos, s.box, charge=s.charge, precision=1)
    eng = mdf.InteractionEngine(sys)
    eng.clearInteraction()
    mdf.ewald_exact(sys, (78, 78, 78), BETA)
    return torch.tensor(sys.forces(), dtype=torch.float64, device="cuda")


def candidates(mdf, order, n=8, seed=11):
    import torch
    base = mdf.optibasis.bspline_initial_basis(order / 2.0, NBIN, order)
    rng = np.random.default_rng(seed + order)
    c = np.tile(base, (n, 1))
    c[1:] += rng.normal(0, 0.1, c[1:].shape)
    return torch.tensor(c, dtype=torch.float64, device="cuda")


def nrel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def noise(f, *args, reps=4):
    """Spread of repeated evaluations (the mesh is summed with FP64 atomics in
    arbitrary order), per candidate; a central difference with step h carries
    up to noise / h of it."""
    v = np.stack([f(*args).cpu().numpy() for _ in range(reps)])
    return v.max(0) - v.min(0)


def test_bspline_basis_is_the_reference_spme(mdf, fluid):
    s, q, r = fluid
    hs = mdf.optibasis.HermiteSPME(s.n, K, s.box, BETA, 2.0, NBIN)
    c = candidates(mdf, 4, n=1)
    out = hs.energy(q, r, c, forces=True)
    sys = mdf.MDSystem(s.pos, s.box, charge=s.charge, precision=1)
    sp = mdf.SPME(sys, K, 4, BETA, "ik")
    eng = mdf.InteractionEngine(sys)
    eng.clearInteraction()
    sys.clear_stats()
    sp.apply()
    E_ref = sys.stats()[mdf.STAT_ELEC_REC]
    F_ref = sys.forces()
    E = out["energy"][0].item()
    F = out["forces"][0].cpu().numpy()
    assert abs(E - E_ref) < 1e-12 * abs(E_ref), (E, E_ref)
    # the Nyquist planes of the spectral derivative are handled differently
    # (zeroed here, FFTW's c2r convention there): a small, bounded difference
    assert nrel(F, F_ref) < 1e-6, nrel(F, F_ref)


@pytest.mark.parametrize("order", [4, 6])
def test_energy_gradients_vs_central_differences(mdf, fluid, order):
    s, q, r = fluid
    hs = mdf.optibasis.HermiteSPME(s.n, K, s.box, BETA, order / 2.0, NBIN)
    c = candidates(mdf, order)
    out = hs.energy(q, r, c, grads=True)
    E = lambda qq, rr, cc: hs.energy(qq, rr, cc)["energy"]  # noqa: E731
    h = 1e-6
    nz = noise(E, q, r, c) / h  # derivative noise bound per candidate
    gc = out["dE_dc"].cpu().numpy()
    fd = np.empty_like(gc)
    for b in range(hs.ncoef):
        cp, cm = c.clone(), c.clone()
        cp[:, b] += h
        cm[:, b] -= h
        fd[:, b] = ((E(q, r, cp) - E(q, r, cm)) / (2 * h)).cpu().numpy()
    for k in range(c.shape[0]):
        err = np.linalg.norm(gc[k] - fd[k])
        assert err <= TOL * np.linalg.norm(fd[k]) + np.sqrt(hs.ncoef) * nz[k], (k, err, np.linalg.norm(fd[k]), nz[k])
    # in q and r the energy (about 1e4, summed over 2.6e5 modes) rounds at the
    # 1e-11 level, which h = 1e-6 would turn into 1e-5 of noise; these use
    # h = 1e-4 (truncation below 1e-8 relative).  The exact comparison of these
    # gradients is the small-system test against the oracle below.
    h = 1e-4
    nz = noise(E, q, r, c) / h
    gq, gr = out["dE_dq"].cpu().numpy(), out["dE_dr"].cpu().numpy()
    for i in (0, 777, 20000):
        qp, qm = q.clone(), q.clone()
        qp[i] += h
        qm[i] -= h
        d = ((E(qp, r, c) - E(qm, r, c)) / (2 * h)).cpu().numpy()
        assert np.all(np.abs(d - gq[:, i]) <= TOL * np.abs(gq[:, i]) + nz), (i, d, gq[:, i], nz)
        # in r only the unperturbed B-spline candidate: a perturbed Hermite basis
        # is C1 with second-derivative jumps at its knots (1/8 grid unit apart),
        # where a central difference is first-order accurate
        for a in range(3):
            rp, rm = r.clone(), r.clone()
            rp[i, a] += h
            rm[i, a] -= h
            d = ((E(q, rp, c[:1]) - E(q, rm, c[:1])) / (2 * h)).cpu().numpy()
            scale = np.abs(gr[0, i]).max()
            assert abs(d[0] - gr[0, i, a]) <= TOL * scale + nz[0], (i, a, d, gr[:, i, a], nz)


@pytest.mark.parametrize("order", [4, 6])
def test_force_error_gradients_vs_central_differences(mdf, fluid, fref, order):
    s, q, r = fluid
    hs = mdf.optibasis.HermiteSPME(s.n, K, s.box, BETA, order / 2.0, NBIN)
    c = candidates(mdf, order)
    out = hs.force_error(q, r, c, fref)
    L = lambda qq, rr, cc: hs.force_error(qq, rr, cc, fref, grads=False)["loss"]  # noqa: E731
    h = 1e-6
    nz = noise(L, q, r, c) / h
    gc = out["dL_dc"].cpu().numpy()
    fd = np.empty_like(gc)
    for b in range(hs.ncoef):
        cp, cm = c.clone(), c.clone()
        cp[:, b] += h
        cm[:, b] -= h
        fd[:, b] = ((L(q, r, cp) - L(q, r, cm)) / (2 * h)).cpu().numpy()
    for k in range(c.shape[0]):
        err = np.linalg.norm(gc[k] - fd[k])
        assert err <= TOL * np.linalg.norm(fd[k]) + np.sqrt(hs.ncoef) * nz[k], (k, err, np.linalg.norm(fd[k]), nz[k])
    gq, gr = out["dL_dq"].cpu().numpy(), out["dL_dr"].cpu().numpy()
    for i in (3, 4242, 19999):
        qp, qm = q.clone(), q.clone()
        qp[i] += h
        qm[i] -= h
        d = ((L(qp, r, c) - L(qm, r, c)) / (2 * h)).cpu().numpy()
        assert np.all(np.abs(d - gq[:, i]) <= TOL * np.abs(gq).max() + nz), (i, d, gq[:, i], nz)
        for a in range(3):
            rp, rm = r.clone(), r.clone()
            rp[i, a] += h
            rm[i, a] -= h
            d = ((L(q, rp, c) - L(q, rm, c)) / (2 * h)).cpu().numpy()
            assert np.all(np.abs(d - gr[:, i, a]) <= TOL * np.abs(gr).max() + nz), (i, a, d, gr[:, i, a], nz)


def test_autograd_functions(mdf, fluid, fref):
    import torch
    from mdforce.optibasis import hermite_spme_energy, hermite_spme_force_error
    s, q, r = fluid
    hs = mdf.optibasis.HermiteSPME(s.n, K, s.box, BETA, 3.0, NBIN)
    c0 = candidates(mdf, 6, n=3)
    ref_e = hs.energy(q, r, c0, grads=True)
    ref_l = hs.force_error(q, r, c0, fref)
    w = torch.tensor([1.0, -2.0, 0.5], dtype=torch.float64, device="cuda")
    for fn, ref, keys in ((lambda a, b, cc: hermite_spme_energy(a, b, cc, hs), ref_e, ("dE_dq", "dE_dr", "dE_dc")),
                          (lambda a, b, cc: hermite_spme_force_error(a, b, cc, fref, hs), ref_l,
                           ("dL_dq", "dL_dr", "dL_dc"))):
        qq = q.clone().requires_grad_(True)
        rr = r.clone().requires_grad_(True)
        cc = c0.clone().requires_grad_(True)
        (w * fn(qq, rr, cc)).sum().backward()
        gq = (w[:, None] * ref[keys[0]]).sum(0)
        gr = (w[:, None, None] * ref[keys[1]]).sum(0)
        gc = w[:, None] * ref[keys[2]]
        # each call sums the mesh with FP64 atomics: equal to rounding
        assert torch.allclose(qq.grad, gq, rtol=1e-9, atol=0)
        assert torch.allclose(rr.grad, gr, rtol=1e-9, atol=1e-12)
        assert torch.allclose(cc.grad, gc, rtol=1e-9, atol=0)


@pytest.mark.parametrize("order", [4, 6])
def test_force_error_near_optibasis_estimate(mdf, fluid, fref, order):
    """The measured RMS reciprocal force error of the B-spline basis and the
    optiBasis estimate of the same basis (homogeneous random charges) agree
    within a factor of three (measured 2.1 for order 6): the estimate is
    statistical, and it takes the continuous transform of the basis (alias 0)
    in the influence function where this SPME takes its integer samples."""
    s, q, r = fluid
    hs = mdf.optibasis.HermiteSPME(s.n, K, s.box, BETA, order / 2.0, NBIN)
    c = candidates(mdf, order, n=1)
    L = hs.force_error(q, r, c, fref, grads=False)["loss"][0].item()
    q2 = float((s.charge ** 2).sum())
    est = mdf.optibasis.IkErrorGPU(order / 2.0, NBIN, BETA, K, q2, s.n, s.box, l_cut=10)
    e, _ = est.evaluate(c.cpu().numpy())
    est_rms = float(e[0]) / mdf.optibasis.CONVERSION
    assert 1.0 / 3.0 < np.sqrt(L) / est_rms < 3.0, (np.sqrt(L), est_rms)


def test_cuda_matches_oracle_small(mdf):
    """The CUDA path against the numpy restatement (oracle/hspme.py, pinned in
    tests/test_hspme_oracle.py) on a small system: energy, forces and every
    gradient of both functionals, two candidates, a bound-0 basis."""
    import torch
    from oracle.hspme import HermiteSPME as Orc
    rng = np.random.default_rng(4)
    n, L = 24, 5.0
    r = rng.uniform(0, L, (n, 3))
    q = rng.uniform(-1, 1, n)
    fref = rng.normal(0, 1, (n, 3))
    for bound0 in (False, True):
        o = Orc((8, 8, 16), (L, L, 2 * L), 1.3, 3.0, 6, bound0=bound0)
        hs = mdf.optibasis.HermiteSPME(n, (8, 8, 16), (L, L, 2 * L), 1.3, 3.0, 6, bound0=bound0)
        base = mdf.optibasis.bspline_initial_basis(3.0, 6, 6, bound0=bound0)
        cs = np.stack([base, base + rng.normal(0, 0.1, base.shape)])
        T = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")  # noqa: E731
        ge = hs.energy(T(q), T(r), T(cs), forces=True, grads=True)
        gl = hs.force_error(T(q), T(r), T(cs), T(fref))
        for k in range(2):
            E, F, dq, dr, dc = o.energy_grad(cs[k], q, r)
            Lo, lq, lr, lc = o.force_error_grad(cs[k], q, r, fref)
            assert abs(ge["energy"][k].item() - E) < 1e-12 * abs(E)
            for got, want in ((ge["forces"][k], F), (ge["dE_dq"][k], dq), (ge["dE_dr"][k], dr), (ge["dE_dc"][k], dc),
                              (gl["dL_dq"][k], lq), (gl["dL_dr"][k], lr), (gl["dL_dc"][k], lc)):
                assert nrel(got.cpu().numpy(), want) < 1e-11, nrel(got.cpu().numpy(), want)
            assert abs(gl["loss"][k].item() - Lo) < 1e-12 * Lo
