"""Parity at the benchmark's own scale: the 65,536-atom liquid-vapour slab
(40 x 40 x 160, adaptive cutoffs 2.5..5.0) in the state bench.py times, read
from tests/golden/slab65536_start.npz (made by make_slab_start.py with the
CPU oracle and the reference's AdaptRCut).  Through the C ABI, against the
oracle:
  - cell indices of the bench's 2.8-sigma cell list, bit-exact;
  - the AdaptRCut estimate on the 41 x 41 x 161 bins of the deposited
    density (error map, rc lattice, bisection indices);
  - per-atom cutoffs assigned from the committed lattice, bit-exact;
  - neighbour sets at rc_i + skin 0.6, bit-exact, order-independent;
  - LJ forces, energy and virial against the FP64 all-pairs oracle.
Both precisions."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
SKIN = 0.6
CELL = 2.8
TOL = {0: 1e-5, 1: 1e-12}  # relative RMS force error, mixed and FP64


@pytest.fixture(scope="module")
def start():
    z = np.load(os.path.join(HERE, "golden", "slab65536_start.npz"))
    return {k: z[k] for k in z.files}


def _system(mdf, start, prec):
    s = mdf.MDSystem(start["pos"].astype(np.float64), start["box"], vel=start["vel"].astype(np.float64),
                     precision=prec)
    mdf.AssignRCut(start["lattice"]).assign(s)
    return s


def _keys(counts, pairs, n):
    rows = np.repeat(np.arange(n, dtype=np.int64), counts)
    return np.sort(rows * n + pairs.astype(np.int64))


@pytest.mark.parametrize("prec", [0, 1])
def test_cells_and_cutoffs_bit_exact(mdf, orc, start, prec):
    s = _system(mdf, start, prec)
    box = start["box"]
    cl = mdf.CellList(s, CELL)
    cl.rebuild()
    nc = cl.ncell()
    assert nc == orc.decide_ncell(box, CELL)[0]
    gp = s.positions()
    if prec == 0:
        _, _, cell = orc.bin_f32(gp.astype(np.float32), box.astype(np.float32), nc)
    else:
        _, _, cell = orc.bin_f64(gp, box, nc)
    assert np.array_equal(cl.cell_index(), cell)
    want = orc.assign_rcut_f32(start["pos"], box, start["lattice"])
    assert np.array_equal(s.rcut(), want)
    assert set(np.unique(want)) <= {2.5, 3.0, 3.5, 4.0, 4.5, 5.0}


def test_adapt_rcut_on_benchmark_bins(mdf, orc, start):
    """Density deposit and the AdaptRCut estimate at target 0.02 on the
    41 x 41 x 161 bins, GPU against the oracle (pinned to the reference's
    AdaptRCut in tests/test_arc_oracle.py)."""
    s = _system(mdf, start, 0)
    box = start["box"]
    arc = mdf.AdaptRCutEstimator(s, refh=1.0, rcmin=2.5, rcmax=5.0, rcstep=0.5)
    assert arc.n == (41, 41, 161)
    arc.clearData()
    arc.deposite()
    arc.update(0.02)
    counts = orc.dp_deposit(s.positions().astype(np.float32), box, arc.n)
    rho = counts / np.prod(box / np.array(arc.n))
    assert np.allclose(arc.profile(), rho, rtol=1e-12, atol=0)
    o = orc.adapt_rcut(box, arc.n, arc.rc_list, rho, 0.02)
    err = arc.error()
    # empty vapour bins of a one-sample profile give NaN errors in the same bins;
    # elsewhere the squared error is a sum of convolutions that nearly cancels in
    # sparse bins, so it is compared with an absolute tolerance on the map's scale
    assert np.array_equal(np.isnan(err), np.isnan(o["error"]))
    scale = np.nanmax(o["error"] ** 2)
    assert np.allclose(err ** 2, o["error"] ** 2, rtol=1e-9, atol=1e-12 * scale, equal_nan=True)
    rc, idx, rerr = arc.rcut()
    assert np.array_equal(idx, o["index"])
    assert np.array_equal(rc, o["rcut"])
    assert np.allclose(rerr ** 2, o["result_error"] ** 2, rtol=1e-9, atol=1e-12 * scale, equal_nan=True)


@pytest.mark.parametrize("prec", [0, 1])
def test_neighbour_sets_bit_exact(mdf, orc, start, prec):
    s = _system(mdf, start, prec)
    box = start["box"]
    cl = mdf.CellList(s, CELL)
    cl.rebuild()
    rc = s.rcut()
    nl = mdf.NeighborList(s, float(rc.max()) + SKIN, SKIN, expansion=1.5)
    nl.fit(s, cl)
    c, p = nl.lists()
    gp = s.positions()
    if prec == 0:
        oc, op = orc.nlist_allpair_f32(gp.astype(np.float32), rc, SKIN, box.astype(np.float32))
    else:
        oc, op = orc.nlist_allpair_f64(gp, rc.astype(np.float64), SKIN, box)
    assert np.array_equal(c, oc), f"list lengths differ at atoms {np.nonzero(c != oc)[0][:10]}"
    assert np.array_equal(_keys(c, p, s.n), _keys(oc, op, s.n))
    assert c.sum() > 1.5e7  # about 2.7e2 entries per atom at these cutoffs


@pytest.mark.parametrize("prec", [0, 1])
def test_forces_vs_allpair_oracle(mdf, orc, start, prec):
    s = _system(mdf, start, prec)
    box = start["box"]
    cl = mdf.CellList(s, CELL)
    cl.rebuild()
    rc = s.rcut()
    nl = mdf.NeighborList(s, float(rc.max()) + SKIN, SKIN, expansion=1.5)
    nl.fit(s, cl)
    eng = mdf.InteractionEngine(s)
    eng.registNonBondedInteraction(1.0, 1.0, 0.0)
    eng.clearInteraction()
    s.clear_stats()
    eng.applyNonBondedInteraction(s, nl, with_stats=True)
    F = s.forces()
    st = s.stats()
    gp = s.positions()
    if prec == 0:
        Fo, so = orc.lj_allpair_f64(gp, rc.astype(np.float64), box, pos32=gp.astype(np.float32),
                                    box32=box.astype(np.float32))
    else:
        Fo, so = orc.lj_allpair_f64(gp, rc.astype(np.float64), box)
    err = float(np.sqrt(((F - Fo) ** 2).sum() / (Fo ** 2).sum()))
    assert err < TOL[prec], err
    assert np.allclose(st[:4], so, rtol=10 * TOL[prec], atol=0), (st[:4], so)
