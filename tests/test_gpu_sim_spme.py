"""GPU tests of the simulation driver with long-range electrostatics: the
engine's real-space Ewald plus the SPME reciprocal part recorded into the
step graph (md_sim_params.spme).  Forces of the first step against the
oracle (LJ all pairs + real-space Ewald + ik SPME), graph vs direct launch,
and the reciprocal energy in the statistics."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BETA, RC, K, ORDER = 1.0, 3.0, (32, 32, 32), 6


@pytest.fixture(scope="module")
def charged(mdf):
    n, L = 512, 10.0
    box = np.array([L, L, L])
    pos = mdf.systems.slab(n, n, box, 2, 0.5 * L, 0.5 * L, 0.9, 5)  # uniform, 0.9 sigma apart
    q = mdf.systems.charges(n, 6)
    return pos, q, box


def make_sim(mdf, pos, q, box, prec, use_graph=True):
    sys = mdf.MDSystem(pos, box, charge=q, precision=prec)
    sys.set_rcut(np.full(len(q), RC, np.float32))
    eng = mdf.InteractionEngine(sys)
    eng.registNonBondedInteraction(1.0, 1.0, 0.0)
    mdf.registCoulomb(eng, BETA)
    sp = mdf.SPME(sys, K, ORDER, BETA, "ik")
    lv = mdf.langevin_params(dt=0.002, temperature=1.0, gamma_t=1.0, seed=3)
    sim = mdf.Simulation(sys, eng, skin=0.3, cell_size=3.3, lv=lv, expansion=2.0, use_graph=use_graph, spme=sp)
    return sys, eng, sp, sim


def test_initial_forces_match_oracle(mdf, orc, charged):
    pos, q, box = charged
    sys, eng, sp, sim = make_sim(mdf, pos, q, box, 1)
    gp = sys.positions()
    F = sys.forces()
    rc = np.full(len(q), RC)
    Flj, _ = orc.lj_allpair_f64(gp, rc, box)
    _, Fd = orc.ewald_dir(gp, q, box, BETA, RC)
    _, Fr = orc.spme_rec(gp, q, box, K, ORDER, BETA, 0)
    Fo = Flj + Fd + Fr
    err = np.sqrt(((F - Fo) ** 2).sum() / (Fo ** 2).sum())
    assert err < 1e-10, err
    st = sys.stats()
    Er, _ = orc.spme_rec(gp, q, box, K, ORDER, BETA, 0)
    assert abs(st[mdf.STAT_ELEC_REC] - Er) < 1e-10 * abs(Er)


def test_graph_and_direct_agree(mdf, charged):
    pos, q, box = charged
    a = make_sim(mdf, pos, q, box, 1, use_graph=True)
    b = make_sim(mdf, pos, q, box, 1, use_graph=False)
    a[3].run(20)
    b[3].run(20)
    d = a[0].positions() - b[0].positions()
    d -= np.round(d / box) * box
    # the charge spread accumulates with atomics: equal up to rounding
    assert np.abs(d).max() < 1e-9


def test_mixed_tracks_fp64(mdf, charged):
    pos, q, box = charged
    a = make_sim(mdf, pos, q, box, 0)
    b = make_sim(mdf, pos, q, box, 1)
    Fa, Fb = a[0].forces(), b[0].forces()
    assert np.sqrt(((Fa - Fb) ** 2).sum() / (Fb ** 2).sum()) < 1e-5
    a[3].run(10)
    b[3].run(10)
    d = a[0].positions() - b[0].positions()
    d -= np.round(d / box) * box
    assert np.abs(d).max() < 1e-3
