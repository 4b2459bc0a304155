"""GPU tests of the long-range force correction (LFC; ForceCorr +
AssignForceCorr of FCR = shortRange.inhomo/template/tools/simulation.fcorr)
through the C ABI: the field against the oracle (pinned to the reference's
own ForceCorr, tests/test_fcorr_oracle.py), the per-atom assignment, its
addition in the non-bonded kernel, and the driver on the fcorr app's
schedule."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def slab_profile(n, L, half, seed=0):
    z = (np.arange(n[2]) + 0.5) * L / n[2]
    rho = np.where(np.abs(z - L / 2) < half, 0.78, 0.02)
    rho = np.ascontiguousarray(np.broadcast_to(rho, n), np.float64)
    return rho * (1 + 0.05 * np.random.default_rng(seed).standard_normal(n))


def slab_system(mdf, prec, n_atoms=2000, box=(12.0, 12.0, 48.0), seed=4):
    box = np.asarray(box, np.float64)
    pos = mdf.systems.slab(n_atoms, int(0.9 * n_atoms), box, 2, 0.5 * box[2], 8.0, 0.85, seed)
    vel = mdf.systems.maxwell(n_atoms, 0.85, seed + 1)
    return mdf.MDSystem(pos, box, vel=vel, precision=prec), box


@pytest.mark.parametrize("rc", [3.5, 5.0])
def test_field_matches_oracle(mdf, orc, rc):
    sys, box = slab_system(mdf, 1)
    fc = mdf.ForceCorr(sys, rc, refh=1.5)
    assert fc.n == orc.dp_bins(box, 1.5)
    rho = slab_profile(fc.n, box[2], 8.0)
    fc.set_profile(rho)
    fc.update()
    re, im = fc.field()
    o = orc.fcorr_field(box, fc.n, rc, rho)
    scale = np.abs(o.real).max()
    assert np.abs(re - o.real).max() < 1e-10 * scale
    assert np.abs(im - o.imag).max() < 1e-10 * scale
    fc.zero()
    re0, im0 = fc.field()
    assert not re0.any() and not im0.any()


@pytest.mark.parametrize("prec", [0, 1])
def test_assign_and_force_addition(mdf, orc, prec):
    sys, box = slab_system(mdf, prec)
    sys.set_rcut(np.full(sys.n, 3.5, np.float32))
    fc = mdf.ForceCorr(sys, 3.5, refh=1.5)
    fc.set_profile(slab_profile(fc.n, box[2], 8.0))
    fc.update()
    re, _ = fc.field()
    cl = mdf.CellList(sys, 3.8)
    cl.rebuild()
    nl = mdf.NeighborList(sys, 3.8, 0.3, expansion=1.5)
    nl.fit(sys, cl)
    fc.assign()
    v = fc.values()
    vo = orc.fcorr_assign(sys.positions(), box, fc.n, re, prec_f32=(prec == 0))
    assert np.array_equal(v, vo)
    assert np.abs(v[:, 2]).max() > 0
    eng = mdf.InteractionEngine(sys)
    eng.registNonBondedInteraction(1.0, 1.0, 0.0)
    eng.clearInteraction(sys)
    eng.applyNonBondedInteraction(sys, nl)
    F0 = sys.forces()
    eng.setForceCorrection(fc)
    eng.clearInteraction(sys)
    eng.applyNonBondedInteraction(sys, nl)
    F1 = sys.forces()
    assert np.abs((F1 - F0) - v).max() < 1e-12 * max(1.0, np.abs(F0).max())


def test_driver_schedule(mdf, orc):
    """fcorr app schedule with assign every 10, samples every 5, update every 20:
    after 21 steps the update (after step 19) has set the field from the samples
    and the assignment of step 20 used it at the current positions."""
    sys, box = slab_system(mdf, 0)
    sys.set_rcut(np.full(sys.n, 3.5, np.float32))
    eng = mdf.InteractionEngine(sys)
    eng.registNonBondedInteraction(1.0, 1.0, 0.0)
    lv = mdf.langevin_params(dt=0.005, temperature=0.85, gamma_t=1.0, seed=3)
    sim = mdf.Simulation(sys, eng, skin=0.3, cell_size=3.8, lv=lv, expansion=1.5)
    fc = mdf.ForceCorr(sys, 3.5, refh=1.5)
    sim.attach_force_corr(fc, assign_every=10, sample_every=5, update_every=20)
    sim.run(20)
    assert not fc.values().any()  # assignments at steps 0 and 10 saw the zero field
    re, _ = fc.field()
    assert np.abs(re[2]).max() > 0
    sim.run(1)
    v = fc.values()
    assert np.array_equal(v, orc.fcorr_assign(sys.positions(), box, fc.n, re, prec_f32=True))
    # the same run without the graph gives the same trajectory up to rounding
    sys2, _ = slab_system(mdf, 0)
    sys2.set_rcut(np.full(sys2.n, 3.5, np.float32))
    eng2 = mdf.InteractionEngine(sys2)
    eng2.registNonBondedInteraction(1.0, 1.0, 0.0)
    sim2 = mdf.Simulation(sys2, eng2, skin=0.3, cell_size=3.8, lv=lv, expansion=1.5, use_graph=False)
    fc2 = mdf.ForceCorr(sys2, 3.5, refh=1.5)
    sim2.attach_force_corr(fc2, assign_every=10, sample_every=5, update_every=20)
    sim2.run(21)
    d = sys.positions() - sys2.positions()
    d -= np.round(d / box) * box
    assert np.abs(d).max() < 1e-4
