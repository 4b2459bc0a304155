"""GPU parity tests of the short-range path through the C ABI:
cell binning (bit-exact), neighbour sets (bit-exact, order-independent),
adaptive-cutoff LJ forces / energy / virial against the FP64 all-pairs
oracle, list overflow handling, and the Langevin driver against the CPU
FP64 oracle trajectory."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# tolerances: relative RMS force error of the mixed path (FP32 pair math,
# compensated / FP64 accumulation) and of the FP64 path against the FP64 oracle
TOL_MIXED = 1e-5
TOL_FP64 = 1e-12


def rel_rms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def as_sets(counts, pairs):
    out, off = [], 0
    for c in counts:
        out.append(np.sort(pairs[off:off + c]))
        off += c
    return out


def assert_same_sets(c1, p1, c2, p2):
    assert np.array_equal(c1, c2), f"count mismatch at {np.nonzero(c1 != c2)[0][:10]}"
    s1, s2 = as_sets(c1, p1), as_sets(c2, p2)
    bad = [i for i in range(len(s1)) if not np.array_equal(s1[i], s2[i])]
    assert not bad, f"neighbour sets differ for atoms {bad[:10]}"


@pytest.fixture(scope="module")
def fluid(mdf):
    return mdf.systems.lj_fluid_fcc()


@pytest.fixture(scope="module")
def small_slab(mdf):
    return mdf.systems.lj_slab(n=8192, box=(20.0, 20.0, 80.0))


def adaptive_rcut(n, seed=0):
    rng = np.random.default_rng(seed)
    return rng.choice(np.arange(2.5, 5.01, 0.5), size=n).astype(np.float32)


@pytest.mark.parametrize("prec", [0, 1])
def test_cell_binning_bit_exact(mdf, orc, fluid, prec):
    rng = np.random.default_rng(5)
    pos = fluid.pos + rng.uniform(-3, 3, size=fluid.pos.shape)  # many atoms outside the box
    pos[0] = [fluid.box[0] * (1 - 1e-9), 0.0, -1e-7]
    sys = mdf.MDSystem(pos, fluid.box, precision=prec)
    cl = mdf.CellList(sys, 2.8)
    cl.rebuild()
    nc = cl.ncell()
    assert nc == orc.decide_ncell(fluid.box, 2.8)[0]
    if prec == 0:
        p, img, cell = orc.bin_f32(pos.astype(np.float32), fluid.box.astype(np.float32), nc)
    else:
        p, img, cell = orc.bin_f64(pos, fluid.box, nc)
    assert np.array_equal(cl.cell_index(), cell)
    gp = sys.positions()
    assert np.array_equal(gp, p.astype(np.float64))
    un = sys.unwrapped_positions()
    L = (fluid.box.astype(np.float32) if prec == 0 else fluid.box).astype(np.float64)
    gimg = np.rint((un - gp) / L).astype(np.int32)
    assert np.array_equal(gimg, img)


@pytest.mark.parametrize("prec", [0, 1])
def test_nlist_uniform_minimage(mdf, orc, fluid, prec):
    sys = mdf.MDSystem(fluid.pos, fluid.box, precision=prec)
    eng = mdf.AssignRCut(np.full((3, 3, 3), 2.5, np.float32))
    eng.uniform(sys, 2.5)
    cl = mdf.CellList(sys, 2.8)
    cl.rebuild()
    nl = mdf.NeighborList(sys, 2.8, 0.3, expansion=2.0)
    nl.rebuild(sys, cl)
    c, p = nl.lists()
    gp = sys.positions()
    if prec == 0:
        oc, op = orc.nlist_allpair_f32(gp.astype(np.float32), np.full(sys.n, 2.5, np.float32), 0.3,
                                       fluid.box.astype(np.float32))
    else:
        oc, op = orc.nlist_allpair_f64(gp, np.full(sys.n, 2.5), 0.3, fluid.box)
    assert_same_sets(c, p, oc, op)
    assert 60 < c.mean() < 100


@pytest.mark.parametrize("prec", [0, 1])
def test_nlist_adaptive_minimage(mdf, orc, small_slab, prec):
    s = small_slab
    rc = adaptive_rcut(s.n)
    sys = mdf.MDSystem(s.pos, s.box, precision=prec)
    sys.set_rcut(rc)
    cl = mdf.CellList(sys, 2.8)
    cl.rebuild()
    nl = mdf.NeighborList(sys, 5.3, 0.3, expansion=3.0)
    nl.fit(sys, cl)
    c, p = nl.lists()
    gp = sys.positions()
    grc = sys.rcut()
    assert np.array_equal(grc, rc)
    if prec == 0:
        oc, op = orc.nlist_allpair_f32(gp.astype(np.float32), grc, 0.3, s.box.astype(np.float32))
    else:
        oc, op = orc.nlist_allpair_f64(gp, grc.astype(np.float64), 0.3, s.box)
    assert_same_sets(c, p, oc, op)


def test_nlist_cellshift_bit_exact(mdf, orc, fluid):
    sys = mdf.MDSystem(fluid.pos, fluid.box, precision=0)
    sys.set_rcut(np.full(sys.n, 2.5, np.float32))
    cl = mdf.CellList(sys, 2.8)
    cl.rebuild()
    nl = mdf.NeighborList(sys, 2.8, 0.3, expansion=2.0, mode=mdf.NL_CELLSHIFT)
    nl.rebuild(sys, cl)
    c, p = nl.lists()
    gp = sys.positions().astype(np.float32)
    nc = cl.ncell()
    _, _, cell = orc.bin_f32(gp, fluid.box.astype(np.float32), nc)
    assert np.array_equal(cell, cl.cell_index())
    oc, op = orc.nlist_cellshift_f32(gp, cell, 2.8, fluid.box.astype(np.float32), nc)
    assert_same_sets(c, p, oc, op)


@pytest.mark.parametrize("prec", [0, 1])
def test_lj_forces_vs_fp64_oracle(mdf, orc, small_slab, prec):
    s = small_slab
    rc = adaptive_rcut(s.n, seed=3)
    sys = mdf.MDSystem(s.pos, s.box, precision=prec)
    sys.set_rcut(rc)
    cl = mdf.CellList(sys, 2.8)
    cl.rebuild()
    nl = mdf.NeighborList(sys, 5.3, 0.3, expansion=3.0)
    nl.fit(sys, cl)
    eng = mdf.InteractionEngine(sys)
    eng.registNonBondedInteraction(1.0, 1.0, 0.0)
    eng.clearInteraction()
    sys.clear_stats()
    eng.applyNonBondedInteraction(sys, nl, with_stats=True)
    F = sys.forces()
    st = sys.stats()
    gp = sys.positions()
    if prec == 0:
        Fo, so = orc.lj_allpair_f64(gp, rc.astype(np.float64), s.box, pos32=gp.astype(np.float32),
                                    box32=s.box.astype(np.float32))
        tol = TOL_MIXED
    else:
        Fo, so = orc.lj_allpair_f64(gp, rc.astype(np.float64), s.box)
        tol = TOL_FP64
    err = rel_rms(F, Fo)
    assert err < tol, err
    assert np.allclose(st[:4], so, rtol=tol * 10, atol=0), (st[:4], so)


def test_nlist_overflow_raises_and_fit_recovers(mdf, fluid):
    sys = mdf.MDSystem(fluid.pos, fluid.box, precision=0)
    sys.set_rcut(np.full(sys.n, 2.5, np.float32))
    cl = mdf.CellList(sys, 2.8)
    cl.rebuild()
    nl = mdf.NeighborList(sys, 2.8, 0.3, expansion=0.2)  # far too small on purpose
    with pytest.raises(mdf.MDExcptShortNeighborList):
        nl.rebuild(sys, cl)
    nl.fit(sys, cl)
    c, _ = nl.lists()
    assert c.max() <= nl.capacity() and c.mean() > 60


def _run_gpu(mdf, s, prec, nsteps, use_graph=True, npt=False, rc=2.5, seed=11, gamma=0.5):
    sys = mdf.MDSystem(s.pos, s.box, vel=s.vel, precision=prec)
    sys.set_rcut(np.full(sys.n, rc, np.float32))
    eng = mdf.InteractionEngine(sys)
    eng.registNonBondedInteraction(1.0, 1.0, 0.0)
    lv = mdf.langevin_params(dt=0.005, temperature=1.0, gamma_t=gamma, seed=seed,
                             tau_p=1.0 if npt else 0.0, kappa_t=0.05 if npt else 0.0,
                             p_ref=(0.0, 0.0, 0.5), npt_dirs=4 if npt else 0)
    sim = mdf.Simulation(sys, eng, skin=0.3, cell_size=2.8, lv=lv, use_graph=use_graph)
    sim.run(nsteps)
    steps, rebuilds, flags = sim.counters()
    return sys, sim, rebuilds


@pytest.mark.parametrize("npt", [False, True])
def test_langevin_fp64_trajectory_matches_oracle(mdf, orc, fluid, npt):
    nsteps = 40
    sys, sim, reb = _run_gpu(mdf, fluid, 1, nsteps, npt=npt)
    out = orc.md_langevin_run(fluid.pos, fluid.vel, fluid.box, nsteps, dt=0.005, temperature=1.0,
                              gamma_t=0.5, skin=0.3, rcut=np.full(fluid.n, 2.5, np.float32), seed=11,
                              tau_p=1.0 if npt else 0.0, kappa_t=0.05 if npt else 0.0,
                              p_ref=(0.0, 0.0, 0.5), npt_dirs=4 if npt else 0)
    assert out["status"] == 0
    assert reb == out["rebuilds"]
    box = sys.box()
    assert np.allclose(box, out["box"], rtol=1e-12, atol=0)
    d = sys.positions() - out["pos"]
    d -= np.round(d / box) * box
    assert np.abs(d).max() < 1e-9
    assert np.abs(sys.velocities() - out["vel"]).max() < 1e-8
    st = sys.stats()
    assert np.allclose(st[:4], out["stats"][:4], rtol=1e-10)


def test_graph_and_direct_launch_agree(mdf, fluid):
    a, _, ra = _run_gpu(mdf, fluid, 0, 30, use_graph=True)
    b, _, rb = _run_gpu(mdf, fluid, 0, 30, use_graph=False)
    assert ra == rb
    assert np.array_equal(a.positions(), b.positions())
    assert np.array_equal(a.velocities(), b.velocities())


def test_mixed_tracks_fp64(mdf, fluid):
    a, _, _ = _run_gpu(mdf, fluid, 0, 20)
    b, _, _ = _run_gpu(mdf, fluid, 1, 20)
    d = a.positions() - b.positions()
    d -= np.round(d / fluid.box) * fluid.box
    assert np.abs(d).max() < 1e-4


def test_langevin_temperature(mdf, fluid):
    # gamma = 2: kinetic relaxation time 1/(2 gamma) = 0.25 tau; 10 tau of
    # equilibration covers the melting of the start lattice
    sys, sim, _ = _run_gpu(mdf, fluid, 0, 2000, gamma=2.0)
    Ts = []
    for _ in range(40):
        sim.run(25)
        st = sys.stats()
        Ts.append(2 * st[mdf.STAT_KINETIC_XX:mdf.STAT_KINETIC_XX + 3].sum() / (3 * sys.n))
    T = np.mean(Ts)
    # BAOAB kinetic temperature is exact for harmonic forces and O(dt^2) here
    assert abs(T - 1.0) < 0.02, T


def test_stream_ordered_stats_rows_match_blocking_reads(mdf, fluid):
    # one row per step queued without a wait equals the blocking read taken
    # after the same step on an identical run (to the order of the FP64
    # block-sum reduction)
    import torch
    a, sa, _ = _run_gpu(mdf, fluid, 0, 0)
    b, sb, _ = _run_gpu(mdf, fluid, 0, 0)
    rows = torch.zeros((5, mdf.STAT_COUNT), dtype=torch.float64).pin_memory().numpy()
    for k in range(5):
        sa.run(1)
        a.stats_async(rows[k])
    a.synchronize()
    for k in range(5):
        sb.run(1)
        assert np.allclose(rows[k], b.stats(), rtol=1e-12, atol=1e-12)
    with pytest.raises(ValueError):
        a.stats_async(np.zeros(3))


def test_system_from_gro_and_back(mdf, fluid, tmp_path):
    # MDSystem::initConfig from a .gro file, a short run, writeHostDataGro
    src = tmp_path / "start.gro"
    mdf.write_gro(src, mdf.GroConf(fluid.pos, fluid.box, fluid.vel, atom_name=["lj"] * fluid.n,
                                   resd_name=["lj"] * fluid.n), "start")
    sys, conf = mdf.system_from_gro(src, precision=1)
    assert np.array_equal(sys.positions(), conf.pos)
    sys.set_rcut(np.full(sys.n, 2.5, np.float32))
    eng = mdf.InteractionEngine(sys)
    eng.registNonBondedInteraction(1.0, 1.0, 0.0)
    lv = mdf.langevin_params(dt=0.005, temperature=1.0, gamma_t=0.5, seed=3)
    sim = mdf.Simulation(sys, eng, skin=0.3, cell_size=2.8, lv=lv)
    sim.run(20)
    out = tmp_path / "confout.gro"
    mdf.write_system_gro(out, sys, conf, step=20, time=0.1)
    back = mdf.read_gro(out)
    assert back.title == "# at time = 0.100000, step = 20"
    assert back.atom_name == conf.atom_name
    assert np.abs(back.pos - sys.positions()).max() < 5e-4 + 1e-4
    assert np.abs(back.vel - sys.velocities()).max() < 5e-5 + 1e-5


TYPED_PAIRS = {(0, 0): (1.0, 1.0, 0.0), (0, 1): (1.5, 0.8, 0.01), (1, 1): (0.5, 0.88, 0.0),
               (0, 2): (0.7, 1.1, -0.02)}  # (1, 2) and (2, 2) never given: no interaction


@pytest.mark.parametrize("prec", [0, 1])
def test_typed_lj_forces_vs_oracle(mdf, orc, small_slab, prec):
    """Several atom types (SystemNonBondedInteraction::add per type pair,
    AtomNBForceTable lookup), adaptive per-atom cutoff, after a cell sort."""
    s = small_slab
    rc = adaptive_rcut(s.n, seed=4)
    types = np.random.default_rng(9).integers(0, 3, s.n)
    sys = mdf.MDSystem(s.pos, s.box, precision=prec, type=types)
    assert np.array_equal(sys.types(), types)
    sys.set_rcut(rc)
    cl = mdf.CellList(sys, 2.8)
    cl.rebuild()
    nl = mdf.NeighborList(sys, 5.3, 0.3, expansion=3.0)
    nl.fit(sys, cl)
    eng = mdf.InteractionEngine(sys)
    for (a, b), v in TYPED_PAIRS.items():
        eng.registNonBondedInteractionPair(a, b, *v)
    eng.clearInteraction()
    sys.clear_stats()
    eng.applyNonBondedInteraction(sys, nl, with_stats=True)
    F, st, gp = sys.forces(), sys.stats(), sys.positions()
    if prec == 0:
        Fo, so = orc.lj_allpair_typed(gp, rc.astype(np.float64), s.box, types, TYPED_PAIRS,
                                      pos32=gp.astype(np.float32), box32=s.box.astype(np.float32))
        tol = TOL_MIXED
    else:
        Fo, so = orc.lj_allpair_typed(gp, rc.astype(np.float64), s.box, types, TYPED_PAIRS)
        tol = TOL_FP64
    assert rel_rms(F, Fo) < tol
    assert np.allclose(st[:4], so, rtol=tol * 10, atol=0), (st[:4], so)


def test_typed_driver_and_arguments(mdf, fluid):
    types = np.arange(fluid.n) % 2
    out = []
    for use_graph in (True, False):
        sys = mdf.MDSystem(fluid.pos, fluid.box, vel=fluid.vel, precision=0, type=types)
        sys.set_rcut(np.full(sys.n, 2.5, np.float32))
        eng = mdf.InteractionEngine(sys)
        eng.registNonBondedInteractionPair(0, 0, 1.0, 1.0)
        eng.registNonBondedInteractionPair(0, 1, 1.2, 0.9)
        eng.registNonBondedInteractionPair(1, 1, 0.8, 1.05)
        lv = mdf.langevin_params(dt=0.005, temperature=1.0, gamma_t=0.5, seed=2)
        sim = mdf.Simulation(sys, eng, skin=0.3, cell_size=2.8, lv=lv, use_graph=use_graph)
        sim.run(50)
        out.append(sys.positions())
        assert np.all(np.isfinite(out[-1]))
        # the types follow their atoms through the sorts
        assert np.array_equal(sys.types(), types)
    assert np.array_equal(out[0], out[1])
    with pytest.raises(mdf.MDExcptBadArgument):
        mdf.MDSystem(fluid.pos, fluid.box, type=np.full(fluid.n, 16))
    with pytest.raises(mdf.MDExcptBadArgument):
        eng.registNonBondedInteractionPair(0, 16, 1.0, 1.0)
    # a system type beyond the interaction table is refused at the force call
    sys = mdf.MDSystem(fluid.pos, fluid.box, precision=0, type=np.arange(fluid.n) % 3)
    sys.set_rcut(np.full(sys.n, 2.5, np.float32))
    eng = mdf.InteractionEngine(sys)
    eng.registNonBondedInteractionPair(0, 1, 1.0, 1.0)
    cl = mdf.CellList(sys, 2.8)
    cl.rebuild()
    nl = mdf.NeighborList(sys, 2.5, 0.3)
    nl.fit(sys, cl)
    with pytest.raises(mdf.MDExcptBadArgument):
        eng.applyNonBondedInteraction(sys, nl)


KIND_PAIRS = {(0, 0): (1.0, 1.0, 0.0), (0, 1): (5, (1.1, 0.95, 0.1, 2.2)), (1, 1): (3, (1.0, 0.95, 1.6)),
              (0, 2): (3, (0.8, 1.0, 0.0)), (2, 2): (1, (0.6, 1.05, -0.01)),
              # capped forms with caps low enough that close pairs of the liquid reach them
              (0, 3): (2, (1.0, 1.0, 0.0, 2.5, 5.0)), (3, 3): (6, (1.0, 1.0, 0.0, 2.2, 4.0)),
              (1, 3): (4, (1.0, 0.95, 1.5, 5.0))}  # (1, 2), (2, 3): none


@pytest.mark.parametrize("prec", [0, 1])
def test_pair_kinds_vs_oracle(mdf, orc, small_slab, prec):
    """Every pair kind of the nbForcePoten dispatch in one typed system: LJ 6-12,
    LJ 6-12 B, CosTail with and without its tail, the three capped forms and
    missing pairs."""
    s = small_slab
    rc = adaptive_rcut(s.n, seed=5)
    types = np.random.default_rng(10).integers(0, 4, s.n)
    sys = mdf.MDSystem(s.pos, s.box, precision=prec, type=types)
    sys.set_rcut(rc)
    cl = mdf.CellList(sys, 2.8)
    cl.rebuild()
    nl = mdf.NeighborList(sys, 5.3, 0.3, expansion=3.0)
    nl.fit(sys, cl)
    eng = mdf.InteractionEngine(sys)
    for (a, b), v in KIND_PAIRS.items():
        if len(v) == 3:
            eng.registNonBondedInteractionPair(a, b, *v)
        else:
            eng.registNonBondedPair(a, b, v[0], v[1])
    eng.clearInteraction()
    sys.clear_stats()
    eng.applyNonBondedInteraction(sys, nl, with_stats=True)
    F, st, gp = sys.forces(), sys.stats(), sys.positions()
    kw = dict(pos32=gp.astype(np.float32), box32=s.box.astype(np.float32)) if prec == 0 else {}
    Fo, so = orc.lj_allpair_typed(gp, rc.astype(np.float64), s.box, types, KIND_PAIRS, **kw)
    tol = TOL_MIXED if prec == 0 else TOL_FP64
    assert rel_rms(F, Fo) < tol
    assert np.allclose(st[:4], so, rtol=tol * 10, atol=0), (st[:4], so)
    with pytest.raises(mdf.MDExcptBadArgument):
        eng.registNonBondedPair(0, 0, 7, (1.0, 1.0))


def test_stats_ring_rows_match_stepwise_reads(mdf, fluid):
    """md_sim_set_stats_ring: the device writes every step's slots into host rows;
    they equal the blocking reads taken after each step of an identical run."""
    import torch
    a, sa, _ = _run_gpu(mdf, fluid, 0, 0)
    b, sb, _ = _run_gpu(mdf, fluid, 0, 0)
    rows = torch.zeros((4, mdf.STAT_COUNT), dtype=torch.float64).pin_memory().numpy()
    sa.set_stats_ring(rows)
    sa.run(6)  # rows wrap: steps 5 and 6 land in rows 0 and 1
    a.synchronize()
    ref = []
    for _ in range(6):
        sb.run(1)
        ref.append(b.stats())
    for row, k in ((2, 2), (3, 3), (0, 4), (1, 5)):
        assert np.allclose(rows[row], ref[k], rtol=1e-12, atol=1e-12)
    # pageable memory is registered by the library for the ring's lifetime
    plain = np.zeros((3, mdf.STAT_COUNT))
    sa.set_stats_ring(plain)
    sa.run(2)
    a.synchronize()
    assert np.allclose(plain[1], a.stats(), rtol=1e-12, atol=1e-12)
    sa.set_stats_ring(None)
    with pytest.raises(ValueError):
        sa.set_stats_ring(np.zeros((3, 4)))


@pytest.mark.parametrize("prec", [0, 1])
def test_statistics_rows_and_finish(mdf, small_slab, prec):
    """with_stats="rows" is the force kernel as the step driver runs it (one row
    of sums per warp, added up later); finishNonBondedStatistics adds the rows
    into the slots exactly as the one-call form does."""
    s = small_slab
    sys = mdf.MDSystem(s.pos, s.box, precision=prec)
    sys.set_rcut(adaptive_rcut(s.n, seed=3))
    cl = mdf.CellList(sys, 2.8)
    cl.rebuild()
    nl = mdf.NeighborList(sys, 5.3, 0.3, expansion=3.0)
    nl.fit(sys, cl)
    eng = mdf.InteractionEngine(sys)
    eng.registNonBondedInteraction(1.0, 1.0, 0.0)
    out = []
    for mode in (True, "rows"):
        eng.clearInteraction()
        sys.clear_stats()
        eng.applyNonBondedInteraction(sys, nl, with_stats=mode)
        if mode == "rows":
            assert not np.any(sys.stats()[:5])  # nothing added yet
            eng.finishNonBondedStatistics(sys)
        out.append((sys.forces(), sys.stats()[:5]))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert np.any(out[0][1])


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("cellshift", [False, True])
def test_fused_rebuild_matches_kernel_chain(mdf, small_slab, prec, use_graph, cellshift):
    """The flag-gated cooperative rebuild (one kernel: cell sort, per-slot
    types, lists) and the chain of kernels give the same trajectory bit for
    bit: adaptive cutoffs, two atom types, Langevin NPT, several rebuilds,
    both list criteria."""
    s = small_slab
    types = np.arange(s.n) % 2
    out = []
    for kind in ("fused", "conditional"):
        sys = mdf.MDSystem(s.pos, s.box, vel=s.vel, precision=prec, type=types)
        sys.set_rcut(adaptive_rcut(s.n, seed=4))
        eng = mdf.InteractionEngine(sys)
        eng.registNonBondedInteractionPair(0, 0, 1.0, 1.0)
        eng.registNonBondedInteractionPair(0, 1, 1.1, 0.95)
        eng.registNonBondedInteractionPair(1, 1, 0.9, 1.05)
        lv = mdf.langevin_params(dt=0.005, temperature=0.85, gamma_t=1.0, seed=9, tau_p=2.0, kappa_t=0.1,
                                 p_ref=(0.0, 0.0, 0.0), npt_dirs=4)
        sim = mdf.Simulation(sys, eng, skin=0.3, cell_size=2.8, lv=lv, use_graph=use_graph, max_rcut=5.0,
                             nl_mode=mdf.NL_CELLSHIFT if cellshift else mdf.NL_MINIMAGE)
        sim.set_rebuild_kind(kind)
        want = kind if (use_graph or kind == "fused") else "gated"
        sim.run(150)
        assert sim.rebuild_kind() == want
        steps, rebuilds, flags = sim.counters()
        out.append((rebuilds, sys.positions(), sys.velocities(), sys.forces(), sys.types(), sys.stats(),
                    sys.box()))
    assert out[0][0] == out[1][0] and out[0][0] >= 3
    for a, b in zip(out[0][1:], out[1][1:]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("with_arc", [False, True])
def test_multi_step_graph_matches_single_steps(mdf, small_slab, with_arc):
    """Simulation.run(n) launches several steps per graph where no host-side
    work falls between them; the trajectory, the statistics and the cutoff
    updates equal those of n single-step runs bit for bit."""
    s = small_slab
    out = []
    for chunked in (False, True):
        sys = mdf.MDSystem(s.pos, s.box, vel=s.vel, precision=0)
        sys.set_rcut(np.full(s.n, 2.5, np.float32))
        eng = mdf.InteractionEngine(sys)
        eng.registNonBondedInteraction(1.0, 1.0, 0.0)
        lv = mdf.langevin_params(dt=0.005, temperature=0.85, gamma_t=1.0, seed=5, tau_p=2.0, kappa_t=0.1,
                                 p_ref=(0.0, 0.0, 0.0), npt_dirs=4)
        sim = mdf.Simulation(sys, eng, skin=0.3, cell_size=2.8, lv=lv, max_rcut=5.0)
        if with_arc:
            arc = mdf.AdaptRCutEstimator(sys, refh=1.0, rcmin=2.5, rcmax=5.0, rcstep=0.5)
            sim.attach_adapt_rcut(arc, sample_every=10, update_every=60, prec=0.02)
        if chunked:
            sim.run(123)
        else:
            for _ in range(123):
                sim.run(1)
        steps, rebuilds, flags = sim.counters()
        assert steps == 123
        out.append((rebuilds, sys.positions(), sys.velocities(), sys.forces(), sys.stats(), sys.box(),
                    sys.rcut()))
    assert out[0][0] == out[1][0] and out[0][0] >= 2
    for a, b in zip(out[0][1:], out[1][1:]):
        assert np.array_equal(a, b)
