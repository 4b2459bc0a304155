"""GPU tests of the adaptive cutoff estimate through the C ABI: k-space
kernel tables, error map, bisection and refinement, tail pressure correction
and the density deposit, each against the CPU oracle (itself pinned to the
reference's AdaptRCut, tests/test_arc_oracle.py); then the driver with the
estimate attached on the reference's schedule."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def slab_profile(n, L=60.0, half=10.0, seed=0):
    z = (np.arange(n[2]) + 0.5) * L / n[2]
    rho = np.where(np.abs(z - L / 2) < half, 0.78, 0.02)
    rho = np.ascontiguousarray(np.broadcast_to(rho, n), np.float64)
    return rho * (1 + 0.05 * np.random.default_rng(seed).standard_normal(n))


@pytest.fixture(scope="module")
def small(mdf):
    box = np.array([20.0, 20.0, 60.0])
    rng = np.random.default_rng(2)
    pos = rng.uniform(0, 1, (500, 3)) * box
    sys = mdf.MDSystem(pos, box, precision=0)
    return sys, box


@pytest.mark.parametrize("nrefine", [0, 2])
def test_arc_gpu_matches_oracle(mdf, orc, small, nrefine):
    sys, box = small
    arc = mdf.AdaptRCutEstimator(sys, refh=4.0, rcmin=2.5, rcmax=5.0, rcstep=0.5)
    n = arc.n
    assert n == orc.dp_bins(box, 4.0)
    rho = slab_profile(n)
    arc.set_profile(rho)
    arc.update(4e-3, nrefine)
    o = orc.adapt_rcut(box, n, arc.rc_list, rho, 4e-3, nrefine=nrefine)
    s1, s2, pck = arc.tables()
    assert np.allclose(s1, o["s1k"], rtol=1e-9, atol=1e-15)
    assert np.allclose(s2, o["s2k"], rtol=1e-9, atol=1e-15)
    assert np.allclose(pck, o["pck"], rtol=1e-6, atol=1e-12)
    err = arc.error()
    assert np.allclose(err, o["error"], rtol=1e-9, atol=0)
    rc, idx, rerr = arc.rcut()
    assert np.array_equal(idx, o["index"])
    assert np.array_equal(rc, o["rcut"])
    p = arc.pressure_correction()
    assert np.allclose(p, o["pcorr"], rtol=1e-6)


def test_density_deposit_matches_oracle(mdf, orc, small):
    sys, box = small
    arc = mdf.AdaptRCutEstimator(sys, refh=2.0, rcmin=2.5, rcmax=5.0, rcstep=0.5)
    arc.clearData()
    arc.deposite()
    arc.deposite()
    arc.update(1e-2)
    pos = sys.positions().astype(np.float32)
    counts = orc.dp_deposit(pos, box, arc.n)
    dv = np.prod(box / np.array(arc.n))
    assert np.allclose(arc.profile(), 2 * counts / (dv * 2))


def test_sim_with_adaptive_cutoff(mdf):
    s = mdf.systems.lj_slab(n=8192, box=(20.0, 20.0, 80.0))
    sys = mdf.MDSystem(s.pos, s.box, vel=s.vel, precision=0)
    sys.set_rcut(np.full(s.n, 2.5, np.float32))
    eng = mdf.InteractionEngine(sys)
    eng.registNonBondedInteraction(1.0, 1.0, 0.0)
    lv = mdf.langevin_params(dt=0.005, temperature=0.85, gamma_t=2.0, seed=3)
    sim = mdf.Simulation(sys, eng, skin=0.3, cell_size=2.8, lv=lv, max_rcut=5.0)
    arc = mdf.AdaptRCutEstimator(sys, refh=1.0, rcmin=2.5, rcmax=5.0, rcstep=0.5)
    sim.attach_adapt_rcut(arc, sample_every=10, update_every=200, prec=0.02)
    sim.run(400)
    steps, rebuilds, flags = sim.counters()
    assert steps == 400 and rebuilds > 0
    rc = sys.rcut()
    assert rc.min() >= 2.5 and rc.max() <= 5.0
    assert len(np.unique(rc)) > 1  # the estimate assigned different cutoffs
    p = sys.stats()
    assert p[mdf.STAT_PRESSURE_CORR_XX] != 0.0
    assert sim.rebuild_kind() == "fused"


def test_pressure_correction_carries_previous_value(mdf, orc, small):
    """PressureCorrection::correction (ENG/src/PressureCorrection.cu:175-211) adds
    each new sum to pxx, pyy, pzz without resetting them and then divides by V,
    so a second update gives p1 / V + (the second profile's own correction)."""
    sys, box = small
    arc = mdf.AdaptRCutEstimator(sys, refh=4.0, rcmin=2.5, rcmax=5.0, rcstep=0.5)
    n = arc.n
    rho1, rho2 = slab_profile(n, seed=0), slab_profile(n, seed=1)
    arc.set_profile(rho1)
    arc.update(4e-3)
    p1 = arc.pressure_correction()
    arc.set_profile(rho2)
    arc.update(4e-3)
    p2 = arc.pressure_correction()
    o1 = orc.adapt_rcut(box, n, arc.rc_list, rho1, 4e-3)["pcorr"]
    o2 = orc.adapt_rcut(box, n, arc.rc_list, rho2, 4e-3)["pcorr"]
    V = float(np.prod(box))
    assert np.allclose(p1, o1, rtol=1e-6)
    assert np.allclose(p2, o1 / V + o2, rtol=1e-6)
    assert not np.allclose(p2, o2, rtol=1e-12, atol=0)  # the carried share is there


def test_box_fixed_at_construction(mdf, orc, small):
    """DensityProfile_PiecewiseConst, AdaptRCut and PressureCorrection take the
    box once at reinit (ENG/src/DensityProfile.cu:22-43, ENG/src/AdaptRCut.cu:
    96-162, ENG/src/PressureCorrection.cu:41-54) and keep it when NPT moves the
    box: after the system's box changes, the kernel tables, the deposit bins,
    the profile normalisation and the estimate are those of the first box."""
    sys, box = small
    pos0 = sys.positions()
    arc = mdf.AdaptRCutEstimator(sys, refh=4.0, rcmin=2.5, rcmax=5.0, rcstep=0.5)
    n = arc.n
    t0 = arc.tables()
    try:
        new_box = box * np.array([1.0, 1.0, 1.03])
        sys.set_box(new_box)
        # deposit: binned and wrapped with the construction box
        arc.clearData()
        arc.deposite()
        pos = sys.positions().astype(np.float32)
        counts = orc.dp_deposit(pos, box, n)
        dv = np.prod(box / np.array(n))
        rho = slab_profile(n)
        arc.set_profile(rho)
        arc.update(4e-3)
        t1 = arc.tables()
        for a, b in zip(t0, t1):
            assert np.array_equal(a, b)
        o = orc.adapt_rcut(box, n, arc.rc_list, rho, 4e-3)
        rc, _, _ = arc.rcut()
        assert np.array_equal(rc, o["rcut"])
        assert np.allclose(arc.pressure_correction(), o["pcorr"], rtol=1e-6)
        # the deposit above, normalised with the construction box
        arc.clearData()
        arc.deposite()
        arc.update(4e-3)
        assert np.allclose(arc.profile(), counts / dv)
    finally:
        sys.set_box(box)
        sys.set_positions(pos0)
