"""Bonded terms and exclusions through the C ABI against the oracle's restatement
of the engine's per-atom gather (oracle_bonded.c, whose force functions equal
the reference headers' own in binary32, test_bonded_oracle.py): forces, the
bonded energy and the virial in both precisions; exclusions removed from the
neighbour list; the driver with bonds."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# binary32 terms summed per atom in binary32 (the reference's arithmetic)
# against the same in the oracle: a few ulp of the largest force
TOL_MIXED = 2e-5
TOL_FP64 = 1e-11


def chains(mdf, n_chain=60, length=12, box=12.0, seed=5):
    """Self-avoiding random-walk chains: bond 0.97, every bead at least 0.9 from
    every earlier bead but its predecessor (periodic), so that no pair force is
    extreme; every bond and angle term type mixed over the chains."""
    rng = np.random.default_rng(seed)
    L = np.full(3, box)
    placed = np.zeros((0, 3))

    def free(q, skip):
        d = placed[:len(placed) - skip] - q if skip else placed - q
        d -= np.round(d / L) * L
        return len(d) == 0 or (d * d).sum(axis=1).min() >= 0.81

    for c in range(n_chain):
        while True:
            chain = [rng.uniform(0, box, 3)]
            if not free(chain[0], 0):
                continue
            base = placed
            ok = True
            while ok and len(chain) < length:
                for _ in range(200):
                    v = rng.normal(size=3)
                    q = chain[-1] + v * (0.97 / np.linalg.norm(v))
                    placed = np.vstack([base] + [np.array(chain)])
                    if free(q, 1):
                        chain.append(q)
                        break
                else:
                    ok = False
            placed = base
            if ok:
                placed = np.vstack([base, np.array(chain)])
                break
    pos = np.mod(placed, box)
    n = len(pos)
    bonds, btype, bparam, angles, atype, aparam = [], [], [], [], [], []
    kinds_b = [(mdf.BOND_FENE, (30.0, 1.5, 0.0)), (mdf.BOND_HARMONIC, (100.0, 1.0, 0.0)),
               (mdf.BOND_FENE2, (20.0, 0.8, 0.95))]
    kinds_a = [(mdf.ANGLE_HARMONIC, (5.0, 1.9, 0.0)), (mdf.ANGLE_COS0, (3.0, 0.0, 0.0))]
    for c in range(n_chain):
        b0 = c * length
        tb, pb = kinds_b[c % 3]
        ta, pa = kinds_a[c % 2]
        for k in range(length - 1):
            bonds.append((b0 + k, b0 + k + 1)); btype.append(tb); bparam.append(pb)
        for k in range(length - 2):
            angles.append((b0 + k, b0 + k + 1, b0 + k + 2)); atype.append(ta); aparam.append(pa)
    return dict(pos=pos, box=np.full(3, box), n=n, bonds=np.array(bonds), btype=np.array(btype),
                bparam=np.array(bparam), angles=np.array(angles), atype=np.array(atype),
                aparam=np.array(aparam))


@pytest.fixture(scope="module")
def poly(mdf):
    return chains(mdf)


def _engine(mdf, s, prec):
    sys = mdf.MDSystem(s["pos"], s["box"], precision=prec)
    eng = mdf.InteractionEngine(sys)
    eng.setBonds(s["bonds"], s["btype"], s["bparam"])
    eng.setAngles(s["angles"], s["atype"], s["aparam"])
    return sys, eng


@pytest.mark.parametrize("prec", [0, 1])
def test_bonded_forces_energy_virial(mdf, orc, poly, prec):
    s = poly
    sys, eng = _engine(mdf, s, prec)
    eng.registBondedInteraction(len(s["bonds"]))
    # sorted into cell order first, so that the slot map is exercised
    cl = mdf.CellList(sys, 2.5)
    cl.rebuild()
    eng.clearInteraction()
    sys.clear_stats()
    eng.applyBondedInteraction(sys)
    F, st = sys.forces(), sys.stats()
    Fo, so = orc.bonded_apply(sys.positions(), s["box"], prec, s["bonds"], s["btype"], s["bparam"],
                              s["angles"], s["atype"], s["aparam"])
    tol = TOL_MIXED if prec == 0 else TOL_FP64
    assert np.abs(F - Fo).max() < tol * np.abs(Fo).max()
    assert abs(st[mdf.STAT_BOND_ENERGY] - so[0]) < tol * abs(so[0])
    vscale = np.abs(so[1:]).max()
    assert np.abs(st[mdf.STAT_VIRIAL_XX:mdf.STAT_VIRIAL_XX + 3] - so[1:]).max() < 10 * tol * vscale
    # Newton's third law of the gathered terms: the total force vanishes
    assert np.abs(F.sum(axis=0)).max() < (1e-3 if prec == 0 else 1e-9) * np.abs(F).max()


def test_bonded_terms_follow_the_atoms_through_sorts(mdf, poly):
    """The same configuration applied before and after a cell sort gives the
    same forces in original order (slot map refreshed by the sort)."""
    s = poly
    sys, eng = _engine(mdf, s, 1)
    eng.clearInteraction()
    eng.applyBondedInteraction(sys)
    F0 = sys.forces()
    cl = mdf.CellList(sys, 2.0)
    cl.rebuild()
    eng.clearInteraction()
    eng.applyBondedInteraction(sys)
    assert np.allclose(sys.forces(), F0, rtol=0, atol=1e-12 * np.abs(F0).max())


@pytest.mark.parametrize("prec", [0, 1])
def test_exclusions_leave_the_neighbour_list(mdf, poly, prec):
    s = poly
    rc = np.full(s["n"], 2.5, np.float32)

    def forces(excl):
        sys = mdf.MDSystem(s["pos"], s["box"], precision=prec)
        sys.set_rcut(rc)
        eng = mdf.InteractionEngine(sys)
        eng.registNonBondedInteraction(1.0, 1.0, 0.0)
        if excl is not None:
            eng.setExclusions(excl)
        cl = mdf.CellList(sys, 2.8)
        cl.rebuild()
        nl = mdf.NeighborList(sys, 2.5, 0.3, expansion=4.0)
        nl.fit(sys, cl)
        eng.clearInteraction()
        eng.applyNonBondedInteraction(sys, nl, with_stats=False)
        return sys, nl

    excl = s["bonds"]
    a, _ = forces(None)
    b, nl = forces(excl)
    # no excluded partner remains in any row (lists in original indices)
    counts, pairs = nl.lists()
    start = np.concatenate([[0], np.cumsum(counts)])
    rows = {i: set(pairs[start[i]:start[i + 1]].tolist()) for i in range(s["n"])}
    assert not any(j in rows[i] or i in rows[j] for i, j in excl)
    Fa, Fb = a.forces(), b.forces()
    # the difference is the LJ force of the excluded pairs (all within 2.5 here)
    pos = a.positions()
    want = np.zeros_like(Fa)
    for i, j in excl:
        d = pos[j] - pos[i]
        d -= np.round(d / s["box"]) * s["box"]
        r2 = d @ d
        if r2 < 2.5 ** 2:
            ri6 = 1.0 / r2 ** 3
            f = 4.0 * (6 * ri6 - 12 * ri6 * ri6) / r2 * d
            want[i] += f
            want[j] -= f
    tol = 1e-5 if prec == 0 else 1e-10
    assert np.abs((Fa - Fb) - want).max() < tol * np.abs(want).max()


def test_driver_with_bonds(mdf, orc, poly):
    """Langevin runs of a bonded melt: graph and direct launch agree bit for bit,
    the bonded energy slot is the one a separate evaluation gives."""
    s = poly
    out = []
    for use_graph in (True, False):
        sys, eng = _engine(mdf, s, 1)
        sys.set_rcut(np.full(s["n"], 2.5, np.float32))
        eng.registNonBondedInteraction(1.0, 1.0, 0.0)
        # 1-3 pairs excluded (bonded pairs keep their LJ repulsion, as in bead-spring melts)
        eng.setExclusions(s["angles"][:, [0, 2]])
        lv = mdf.langevin_params(dt=0.002, temperature=1.0, gamma_t=1.0, seed=7)
        sim = mdf.Simulation(sys, eng, skin=0.3, cell_size=2.8, lv=lv, use_graph=use_graph)
        sim.run(200)
        out.append((sys.positions(), sys.stats()))
        assert np.all(np.isfinite(out[-1][0]))
    assert np.array_equal(out[0][0], out[1][0])
    e_run = out[0][1][mdf.STAT_BOND_ENERGY]
    _, so = orc.bonded_apply(out[0][0], s["box"], 1, s["bonds"], s["btype"], s["bparam"], s["angles"],
                             s["atype"], s["aparam"])
    # the slot holds the energy of the last force evaluation, at the positions
    # before the last drift; a loose comparison
    assert e_run > 0 and abs(e_run - so[0]) < 0.05 * abs(so[0])


def test_bad_topologies_are_rejected(mdf, poly):
    s = poly
    sys, eng = _engine(mdf, s, 0)
    with pytest.raises(mdf.MDExcptBadArgument):
        eng.setBonds([[0, 0]], mdf.BOND_HARMONIC, (1.0, 1.0))
    with pytest.raises(mdf.MDExcptBadArgument):
        eng.setBonds([[0, s["n"]]], mdf.BOND_HARMONIC, (1.0, 1.0))
    with pytest.raises(mdf.MDExcptBadArgument):
        eng.setBonds([[0, 1]], 12345, (1.0, 1.0))
    with pytest.raises(mdf.MDExcptBadArgument):
        eng.setBonds([[0, 1]], mdf.BOND_FENE, (1.0, -1.0))
    with pytest.raises(mdf.MDExcptBadArgument):
        eng.setAngles([[0, 1, 1]], mdf.ANGLE_HARMONIC, (1.0, 1.0))
    with pytest.raises(mdf.MDExcptBadArgument):
        eng.setExclusions([[3, 3]])
    with pytest.raises(mdf.MDExcptBadArgument):
        eng.registBondedInteraction(3)


def test_topology_path_equals_direct_lists(mdf, poly):
    """Molecules and copy numbers (Topology::System) give the same bonded forces
    as the expanded lists handed over directly."""
    s = poly
    t = mdf.topology
    length = 12
    chain = t.Molecule("chain")
    for _ in range(length):
        chain.pushAtom(t.Atom("B", 0, 1.0, 0.0))
    for k in range(length - 1):
        chain.addBond(t.Bond(k, k + 1, mdf.BOND_FENE, (30.0, 1.5)))
    for k in range(length - 2):
        chain.addAngle(t.Angle(k, k + 1, k + 2, mdf.ANGLE_COS0, (3.0,)))
    top = t.System()
    top.addMolecules(chain, s["n"] // length)
    a = mdf.MDSystem(s["pos"], s["box"], precision=1)
    ea = mdf.InteractionEngine(a)
    e = t.registBondedInteraction(ea, top)
    t.initTopology(a, top)
    ea.clearInteraction()
    ea.applyBondedInteraction(a)
    b = mdf.MDSystem(s["pos"], s["box"], precision=1)
    eb = mdf.InteractionEngine(b)
    eb.setBonds(e["bonds"], mdf.BOND_FENE, (30.0, 1.5))
    eb.setAngles(e["angles"], mdf.ANGLE_COS0, (3.0,))
    eb.clearInteraction()
    eb.applyBondedInteraction(b)
    assert np.array_equal(a.forces(), b.forces())


def test_init_topology_sets_masses(mdf, poly):
    """initTopology copies each atom's mass, charge and type from the topology,
    as MDSystem::initTopology does; masses reach the integrator as 1/m."""
    s = poly
    t = mdf.topology
    mol = t.Molecule("pair")
    mol.pushAtom(t.Atom("A", 0, 2.0, 0.5))
    mol.pushAtom(t.Atom("B", 1, 0.5, -0.5))
    top = t.System()
    top.addMolecules(mol, s["n"] // 2)
    for prec in (0, 1):
        a = mdf.MDSystem(s["pos"][: 2 * (s["n"] // 2)], s["box"], precision=prec)
        t.initTopology(a, top)
        want = np.tile([2.0, 0.5], s["n"] // 2)
        assert np.allclose(a.masses(), want, rtol=1e-7)
        assert np.array_equal(a.types(), np.tile([0, 1], s["n"] // 2))
        assert np.allclose(a.charges(), np.tile([0.5, -0.5], s["n"] // 2))
        with pytest.raises(mdf.MDExcptBadArgument):
            a.set_masses(np.zeros(a.n))
