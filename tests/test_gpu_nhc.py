"""GPU tests of the Nose-Hoover chain velocity-Verlet path (md_nhc_*, the
integrator of ENG/app/lj.nhc-xtc.cu) through the C ABI: manual stepping and
the graph-captured driver against the literal CPU FP64 restatement of the
reference step (oracle orc_md_nhc_run), run splitting, and conservation of
E + K + H_NHC."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT, T, TAU, SKIN = 0.005, 1.0, 0.5, 0.3


@pytest.fixture(scope="module")
def fluid(mdf):
    return mdf.systems.lj_fluid_fcc()


def shift25():
    return -4.0 * (2.5 ** -12 - 2.5 ** -6)


def make_system(mdf, s, prec):
    sys = mdf.MDSystem(s.pos, s.box, vel=s.vel, precision=prec)
    sys.set_rcut(np.full(s.n, 2.5, np.float32))
    eng = mdf.InteractionEngine(sys)
    eng.registNonBondedInteraction(1.0, 1.0, shift25())
    return sys, eng


def oracle_run(orc, s, nsteps):
    out = orc.md_nhc_run(s.pos, s.vel, s.box, nsteps, dt=DT, temperature=T, tau_t=TAU, skin=SKIN,
                         rcut=np.full(s.n, 2.5, np.float32), shift=shift25(), cap=256)
    assert out["status"] == 0
    return out


def compare(sys, out, box, tol=1e-9):
    d = sys.positions() - out["pos"]
    d -= np.round(d / box) * box
    assert np.abs(d).max() < tol
    assert np.abs(sys.velocities() - out["vel"]).max() < tol


def test_manual_steps_match_oracle(mdf, orc, fluid):
    nsteps = 20
    sys, eng = make_system(mdf, fluid, 1)
    cl = mdf.CellList(sys, 2.8)
    cl.rebuild()
    nl = mdf.NeighborList(sys, 2.8, SKIN, expansion=2.0)
    nl.fit(sys, cl)
    eng.clearInteraction()
    eng.applyNonBondedInteraction(sys, nl, with_stats=True)
    nhc = mdf.NoseHoover_Chains2(sys, T, TAU)
    rebuilds = 0
    for _ in range(nsteps):
        nhc.step1(DT, nl)
        if nl.max_displacement() > 0.5 * SKIN:
            cl.rebuild()
            nl.rebuild(sys, cl)
            rebuilds += 1
        sys.clear_stats()
        eng.clearInteraction()
        eng.applyNonBondedInteraction(sys, nl, with_stats=True)
        nhc.step2(DT)
    out = oracle_run(orc, fluid, nsteps)
    assert rebuilds == out["rebuilds"]
    compare(sys, out, fluid.box)
    st = nhc.state()
    assert np.allclose(st, out["nhc"], rtol=1e-10, atol=1e-12)
    k = sys.stats()[mdf.STAT_KINETIC_XX:mdf.STAT_KINETIC_XX + 3]
    assert np.allclose(k, out["stats"][4:7], rtol=1e-10)


def run_driver(mdf, s, prec, chunks, use_graph=True):
    sys, eng = make_system(mdf, s, prec)
    lv = mdf.langevin_params(dt=DT, temperature=T, gamma_t=0.0, seed=1)
    sim = mdf.Simulation(sys, eng, skin=SKIN, cell_size=2.8, lv=lv, expansion=2.0, use_graph=use_graph,
                         integrator="nhc", nhc_tau=TAU)
    for c in chunks:
        sim.run(c)
    return sys, sim


def test_driver_matches_oracle(mdf, orc, fluid):
    sys, sim = run_driver(mdf, fluid, 1, [20])
    out = oracle_run(orc, fluid, 20)
    _, reb, _ = sim.counters()
    assert reb == out["rebuilds"]
    compare(sys, out, fluid.box)
    assert np.allclose(sim.nhc_state(), out["nhc"], rtol=1e-10, atol=1e-12)
    st = sys.stats()
    assert np.allclose(st[mdf.STAT_KINETIC_XX:mdf.STAT_KINETIC_XX + 3], out["stats"][4:7], rtol=1e-10)
    assert np.allclose(st[:4], out["stats"][:4], rtol=1e-10)


def test_driver_run_splitting_and_direct_launch(mdf, fluid):
    a, sa = run_driver(mdf, fluid, 1, [20])
    b, sb = run_driver(mdf, fluid, 1, [7, 13])
    c, sc = run_driver(mdf, fluid, 1, [20], use_graph=False)
    for x in (b, c):
        d = a.positions() - x.positions()
        d -= np.round(d / fluid.box) * fluid.box
        assert np.abs(d).max() < 1e-11
        assert np.abs(a.velocities() - x.velocities()).max() < 1e-11
    assert np.allclose(sa.nhc_state(), sb.nhc_state(), rtol=1e-11)
    assert np.array_equal(a.velocities(), c.velocities())


def test_isobaric_operators_match_oracle(mdf, orc, fluid):
    """NoseHoover_Chains2_Isobaric operators composed into the MTK step
    (L_CP L_v L_r L_box | forces | L_v L_CP), list rebuilt every step, FP64."""
    nsteps, dt, Pref, tauP = 15, 0.002, 1.0, 1.0
    sys, eng = make_system(mdf, fluid, 1)
    cl = mdf.CellList(sys, 2.8)
    nl = mdf.NeighborList(sys, 2.8, SKIN, expansion=2.0)

    def forces():
        cl.rebuild()
        nl.fit(sys, cl)
        eng.clearInteraction()
        sys.clear_stats()
        eng.applyNonBondedInteraction(sys, nl, with_stats=True)

    forces()
    npt = mdf.NoseHoover_Chains2_Isobaric(sys, T, TAU, Pref, tauP, 0.0)
    for _ in range(nsteps):
        npt.operator_L_CP(0.5 * dt)
        npt.operator_L_v(0.5 * dt)
        npt.operator_L_r(dt)
        npt.operator_L_box(dt)
        forces()
        npt.operator_L_v(0.5 * dt)
        npt.operator_L_CP(0.5 * dt)
    out = orc.md_nhc_npt_run(fluid.pos, fluid.vel, fluid.box, nsteps, dt=dt, temperature=T, tau_t=TAU,
                             p_ref=Pref, tau_p=tauP, skin=SKIN, rcut=np.full(fluid.n, 2.5, np.float32),
                             shift=shift25(), cap=256)
    assert out["status"] == 0
    box = sys.box()
    assert np.allclose(box, out["box"], rtol=1e-11, atol=0)
    compare(sys, out, box)
    assert np.allclose(npt.state(), out["state"], rtol=1e-10, atol=1e-12)
    k = sys.stats()[mdf.STAT_KINETIC_XX:mdf.STAT_KINETIC_XX + 3]
    assert np.allclose(k, out["stats"][4:7], rtol=1e-10)


def test_mixed_conserves_extended_energy(mdf, fluid):
    sys, sim = run_driver(mdf, fluid, 0, [200])
    vals = []
    for _ in range(10):
        sim.run(100)
        st = sys.stats()
        vals.append(st[mdf.STAT_NB_ENERGY] + st[mdf.STAT_KINETIC_XX:mdf.STAT_KINETIC_XX + 3].sum()
                    + sim.nhc_state()[4])
    vals = np.array(vals)
    # the shifted potential at rc 2.5 with skin 0.3 and dt 0.005: drift well
    # below 1e-3 of the magnitude over 1000 steps
    assert np.abs(vals - vals[0]).max() < 1e-3 * abs(vals[0]), vals
