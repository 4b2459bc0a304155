"""The grid barrier of the fused rebuild waits a bounded time: when a block
never arrives (a wait that nothing ends), the other blocks give up after
the limit, set the timeout flag and return, and the GPU context and the
system stay usable; a normal barrier completes without the flag."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fluid(mdf):
    return mdf.systems.lj_fluid_fcc()


def test_barrier_completes(mdf, fluid):
    sys = mdf.MDSystem(fluid.pos, fluid.box, vel=fluid.vel, precision=0)
    for _ in range(3):
        assert not mdf.check_grid_barrier(sys, skip_block=-1, limit_s=1.0)


@pytest.mark.parametrize("skip", [0, 7])
def test_barrier_wait_is_bounded(mdf, fluid, skip):
    sys = mdf.MDSystem(fluid.pos, fluid.box, vel=fluid.vel, precision=0)
    t0 = time.perf_counter()
    assert mdf.check_grid_barrier(sys, skip_block=skip, limit_s=0.05)
    assert time.perf_counter() - t0 < 5.0
    # the flag is cleared and the counter realigned: a normal barrier passes
    assert not mdf.check_grid_barrier(sys, skip_block=-1, limit_s=1.0)
    # and the driver, whose rebuild uses the barrier, runs on the same system
    sys.set_rcut(np.full(sys.n, 2.5, np.float32))
    eng = mdf.InteractionEngine(sys)
    eng.registNonBondedInteraction(1.0, 1.0, 0.0)
    lv = mdf.langevin_params(dt=0.005, temperature=1.0, gamma_t=0.5, seed=3)
    sim = mdf.Simulation(sys, eng, skin=0.3, cell_size=2.8, lv=lv)
    sim.run(100)
    steps, rebuilds, flags = sim.counters()
    assert steps == 100 and rebuilds > 0
    assert np.all(np.isfinite(sys.positions()))


def test_barrier_arguments(mdf, fluid):
    sys = mdf.MDSystem(fluid.pos, fluid.box, precision=0)
    with pytest.raises(mdf.MDExcptBadArgument):
        mdf.check_grid_barrier(sys, skip_block=-1, limit_s=0.0)
    with pytest.raises(mdf.MDExcptBadArgument):
        mdf.check_grid_barrier(sys, skip_block=1 << 20, limit_s=0.05)
