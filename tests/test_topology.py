"""The topology mirror (Topology::Molecule / System and their expansion into the
global lists that SystemBondedInteraction, BondedInteractionList and
ExclusionList build): host logic only."""
import numpy as np
import pytest


def water_like(mdf):
    t = mdf.topology
    m = t.Molecule("W")
    m.pushAtom(t.Atom("O", 0, 16.0, -0.8))
    m.pushAtom(t.Atom("H1", 1, 1.0, 0.4))
    m.pushAtom(t.Atom("H2", 1, 1.0, 0.4))
    m.addBond(t.Bond(0, 1, mdf.BOND_HARMONIC, (500.0, 0.1)))
    m.addBond(t.Bond(0, 2, mdf.BOND_HARMONIC, (500.0, 0.1)))
    m.addAngle(t.Angle(1, 0, 2, mdf.ANGLE_HARMONIC, (50.0, 1.91)))
    m.addExclusion(t.Exclusion(1, 2))
    return m


def test_expansion_follows_the_copy_order(mdf):
    t = mdf.topology
    chain = t.Molecule("C")
    for _ in range(4):
        chain.pushAtom(t.Atom("B", 2, 1.0, 0.0))
    for k in range(3):
        chain.addBond(t.Bond(k, k + 1, mdf.BOND_FENE, (30.0, 1.5)))
    top = t.System()
    top.addMolecules(water_like(mdf), 2)
    top.addMolecules(chain, 3)
    assert top.indexShift == [0, 6, 18] and top.numAtom() == 18
    e = top.expand()
    assert e["type"].tolist() == [0, 1, 1, 0, 1, 1] + [2] * 12
    assert np.allclose(e["charge"][:6], [-0.8, 0.4, 0.4] * 2)
    assert e["bonds"].tolist()[:4] == [[0, 1], [0, 2], [3, 4], [3, 5]]
    assert e["bonds"].tolist()[4:7] == [[6, 7], [7, 8], [8, 9]]
    assert e["bonds"].shape == (4 + 9, 2) and e["btype"].tolist()[-1] == mdf.BOND_FENE
    assert e["angles"].tolist() == [[1, 0, 2], [4, 3, 5]]
    assert e["exclusions"].tolist() == [[1, 2], [4, 5]]
    assert e["bparam"].shape == (13, 3) and e["bparam"][5].tolist() == [30.0, 1.5, 0.0]


def test_bad_indices_are_rejected(mdf):
    t = mdf.topology
    m = t.Molecule("M")
    m.pushAtom(t.Atom())
    with pytest.raises(ValueError):
        m.addBond(t.Bond(0, 1))
