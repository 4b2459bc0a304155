"""Statistical acceptance of the Langevin integrator, the only parity a path
with no reference code can have (langevin.npt/writedown/paper.tex:355-369,
586-600 give the equations of motion with friction gamma_T and noise variance
2 k_B T gamma_T, and the box equations with gamma_P and the piston mass):

  - NVT, ideal gas (forces switched off): the velocity autocorrelation decays
    as exp(-gamma_T t), since the friction and noise are the only forces; the
    velocity components are Gaussian with variance k_B T / m (second and
    fourth moments, skewness);
  - NPT along z with P_zz = 0 (x, y fixed, the slab benchmark's barostat) on
    an LJ liquid: the block-averaged <P_zz> is 0 within 3 sigma over 25 blocks.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_nvt_ideal_gas_vacf_and_moments(mdf):
    n, L, T, gamma, dt = 4096, 20.0, 1.5, 0.8, 0.005
    rng = np.random.default_rng(7)
    pos = rng.uniform(0, L, (n, 3))
    vel = mdf.systems.maxwell(n, T, 9)
    box = np.array([L, L, L])
    sys = mdf.MDSystem(pos, box, vel=vel, precision=1)
    sys.set_rcut(np.full(n, 2.5, np.float32))
    eng = mdf.InteractionEngine(sys)
    eng.registNonBondedInteraction(0.0, 1.0, 0.0)  # no forces: the Langevin terms alone
    lv = mdf.langevin_params(dt=dt, temperature=T, gamma_t=gamma, seed=5)
    sim = mdf.Simulation(sys, eng, skin=0.3, cell_size=2.8, lv=lv)
    sim.run(500)
    every, nsnap = 25, 240
    snaps = np.empty((nsnap, n, 3))
    for k in range(nsnap):
        sim.run(every)
        snaps[k] = sys.velocities()
    v = snaps.reshape(-1)
    # Maxwell-Boltzmann moments (m = 1): <v^2> = T, <v^4> = 3 T^2, no skew
    m2 = float((v ** 2).mean())
    assert abs(m2 / T - 1) < 0.01, m2
    assert abs(float((v ** 4).mean()) / (3 * T * T) - 1) < 0.03
    assert abs(float((v ** 3).mean()) / T ** 1.5) < 0.02
    # velocity autocorrelation over lags of 25 steps: exactly (exp(-gamma dt))^(25 l)
    lags = np.arange(0, 13)
    C = np.array([(snaps[: nsnap - l] * snaps[l:]).sum(-1).mean() for l in lags]) / (3 * m2)
    t = lags * every * dt
    want = np.exp(-gamma * t)
    assert np.all(np.abs(C - want) < 0.01), np.c_[t, C, want]
    # decay rate from a least-squares fit of log C over the lags where C > 0.1
    ok = C > 0.1
    g_fit = -np.polyfit(t[ok], np.log(C[ok]), 1)[0]
    assert abs(g_fit / gamma - 1) < 0.03, g_fit


def test_npt_pzz_zero_block_average(mdf):
    n, rho, T = 4000, 0.78, 0.7
    L = (n / rho) ** (1.0 / 3.0)
    box = np.array([L, L, L])
    pos = mdf.systems.slab(n, n, box, 2, 0.5 * L, 0.5 * L + 1.0, 0.8, 3)
    rc = 2.5
    shift = -4.0 * (rc ** -12 - rc ** -6)

    def build(p, v, npt, gamma, seed):
        sys = mdf.MDSystem(p, box if npt is None else npt, vel=v, precision=0)
        sys.set_rcut(np.full(n, rc, np.float32))
        eng = mdf.InteractionEngine(sys)
        eng.registNonBondedInteraction(1.0, 1.0, shift)
        lv = mdf.langevin_params(dt=0.005, temperature=T, gamma_t=gamma, seed=seed,
                                 tau_p=1.0 if npt is not None else 0.0, kappa_t=0.05 if npt is not None else 0.0,
                                 p_ref=(0.0, 0.0, 0.0), npt_dirs=4 if npt is not None else 0)
        return sys, eng, mdf.Simulation(sys, eng, skin=0.3, cell_size=2.8, lv=lv)

    # relax the random start (0.8 sigma contacts) at fixed volume
    sys0, _, sim0 = build(pos, mdf.systems.maxwell(n, T, 4), None, 2.0, 11)
    sim0.run(1500)
    p0, v0 = sys0.positions(), sys0.velocities()
    del sim0, sys0
    sys, eng, sim = build(p0, v0, box, 1.0, 12)
    sim.run(4000)  # the box relaxes to P_zz = 0
    nblock, per_block, every = 25, 80, 10
    pzz = np.empty((nblock, per_block))
    lz = np.empty(nblock * per_block)
    for b in range(nblock):
        for k in range(per_block):
            sim.run(every)
            pzz[b, k] = sys.pressure()[2]
            lz[b * per_block + k] = sys.box()[2]
    means = pzz.mean(1)
    mean = float(means.mean())
    sem = float(means.std(ddof=1) / np.sqrt(nblock))
    assert abs(mean) < 3 * sem, (mean, sem)
    assert sem < 0.02  # the test resolves the pressure
    # x and y stay fixed, z moved and fluctuates
    b = sys.box()
    assert b[0] == box[0] and b[1] == box[1]
    assert lz.std() > 0 and abs(lz.mean() - L) > 0.05
