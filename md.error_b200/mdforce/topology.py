"""Molecular topology in the shape of the reference's Topology namespace
(shortRange.inhomo/template/tools/simulation.hetero.cutoff/include/Topology.h:21-165):
atoms with type, mass and charge; bonds, angles and exclusions by index inside a
molecule; a system of molecule kinds with copy numbers.  expand() lays the copies
out in order (the reference's indexShift), giving the per-atom arrays that
MDSystem::initTopology fills and the global term lists that
SystemBondedInteraction::reinit / BondedInteractionList / ExclusionList build
(src/SystemBondedInteraction.cu:100-230, src/BondedInteractionList.cu:40-90,
src/ExclusionList.cu:175-200).  Host code only."""
from dataclasses import dataclass, field

import numpy as np

from .core import ANGLE_COS0, ANGLE_HARMONIC, BOND_FENE, BOND_FENE2, BOND_HARMONIC  # noqa: F401


@dataclass
class Atom:
    name: str = ""
    type: int = 0
    mass: float = 1.0
    charge: float = 0.0

    def setProperty(self, mass, charge):
        self.mass, self.charge = float(mass), float(charge)


@dataclass
class Bond:
    atom0: int
    atom1: int
    kind: int = BOND_HARMONIC
    params: tuple = (0.0, 0.0)

    def specifyInteraction(self, atom0, atom1, kind, params):
        self.atom0, self.atom1, self.kind, self.params = int(atom0), int(atom1), int(kind), tuple(params)


@dataclass
class Angle:
    edge0: int
    center: int
    edge1: int
    kind: int = ANGLE_HARMONIC
    params: tuple = (0.0, 0.0)


@dataclass
class Exclusion:
    atom0: int
    atom1: int


@dataclass
class Molecule:
    name: str = ""
    atoms: list = field(default_factory=list)
    bonds: list = field(default_factory=list)
    angles: list = field(default_factory=list)
    exclusions: list = field(default_factory=list)

    def pushAtom(self, a):
        self.atoms.append(a)

    def addBond(self, b):
        self._check(b.atom0, b.atom1)
        self.bonds.append(b)

    def addAngle(self, a):
        self._check(a.edge0, a.center, a.edge1)
        self.angles.append(a)

    def addExclusion(self, x):
        self._check(x.atom0, x.atom1)
        self.exclusions.append(x)

    def size(self):
        return len(self.atoms)

    def _check(self, *idx):
        for i in idx:
            if not 0 <= i < len(self.atoms):
                raise ValueError(f"molecule {self.name!r}: atom index {i} outside 0..{len(self.atoms) - 1}")


class System:
    """Topology::System: molecule kinds and their copy numbers, in the order the
    configuration lists them."""

    def __init__(self):
        self.molecules, self.numbers, self.indexShift = [], [], [0]

    def addMolecules(self, mol, number):
        self.molecules.append(mol)
        self.numbers.append(int(number))
        self.indexShift.append(self.indexShift[-1] + mol.size() * int(number))

    def numAtom(self):
        return self.indexShift[-1]

    def expand(self):
        """Per-atom type, mass, charge and the global bond / angle / exclusion lists
        (atoms numbered molecule copy by copy)."""
        n = self.numAtom()
        out = dict(type=np.zeros(n, np.int32), mass=np.ones(n), charge=np.zeros(n),
                   bonds=[], btype=[], bparam=[], angles=[], atype=[], aparam=[], exclusions=[])
        for mol, num, s0 in zip(self.molecules, self.numbers, self.indexShift):
            m = mol.size()
            for c in range(num):
                base = s0 + c * m
                for k, a in enumerate(mol.atoms):
                    out["type"][base + k] = a.type
                    out["mass"][base + k] = a.mass
                    out["charge"][base + k] = a.charge
                for b in mol.bonds:
                    out["bonds"].append((base + b.atom0, base + b.atom1))
                    out["btype"].append(b.kind)
                    out["bparam"].append(tuple(b.params) + (0.0,) * (3 - len(b.params)))
                for a in mol.angles:
                    out["angles"].append((base + a.edge0, base + a.center, base + a.edge1))
                    out["atype"].append(a.kind)
                    out["aparam"].append(tuple(a.params) + (0.0,) * (3 - len(a.params)))
                for x in mol.exclusions:
                    out["exclusions"].append((base + x.atom0, base + x.atom1))
        for k in ("bonds", "angles", "exclusions"):
            w = 2 if k != "angles" else 3
            out[k] = np.array(out[k], np.int32).reshape(-1, w)
        for k in ("btype", "atype"):
            out[k] = np.array(out[k], np.int32)
        for k in ("bparam", "aparam"):
            out[k] = np.array(out[k], np.float64).reshape(-1, 3)
        return out


def initTopology(sys, top):
    """MDSystem::initTopology (shortRange.inhomo/template/tools.collision/cal.real.error/
    src/MDSystem_interface.cu:116-133): the system's types, masses and charges from the
    topology."""
    e = top.expand()
    if e["type"].shape[0] != sys.n:
        raise ValueError(f"topology has {e['type'].shape[0]} atoms, the system {sys.n}")
    sys.set_types(e["type"])
    sys.set_masses(e["mass"])
    sys.set_charges(e["charge"])
    return e


def registBondedInteraction(engine, top):
    """SystemBondedInteraction(sysTop) + BondedInteractionList + ExclusionList:
    every bond, angle and exclusion of the topology given to the engine."""
    e = top.expand()
    engine.setBonds(e["bonds"], e["btype"], e["bparam"])
    engine.setAngles(e["angles"], e["atype"], e["aparam"])
    engine.setExclusions(e["exclusions"])
    engine.registBondedInteraction(len(e["bonds"]))
    return e
