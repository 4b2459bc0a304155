"""CPU tests: the C ABI library loads and exports every declared symbol; the
oracle's binary32 restatements are pinned against hand-derived known answers
and published Philox vectors; the synthetic generators meet their spec."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\*?\s+\*?(md_[a-z_0-9]+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(mdf):
    import ctypes
    names = declared_functions()
    assert len(names) > 40
    lib = ctypes.CDLL(mdf.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes table covers them all
    assert set(names) <= set(mdf.EXPORTED), sorted(set(names) - set(mdf.EXPORTED))


def test_version_and_device_count(mdf):
    assert "sm_100a" in mdf.__version__
    assert mdf.device_count() >= 0


def test_philox_known_answers(orc):
    # Random123 (Salmon et al., SC'11) known-answer vectors for philox4x32-10
    kat = [
        ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
        ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
        ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
         (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
    ]
    for ctr, key, want in kat:
        assert tuple(int(x) for x in orc.philox4x32_10(ctr, key)) == want


def test_normals_moments(orc):
    z = np.array([orc.normals4(7, s, i) for s in range(1, 200) for i in range(50)]).ravel()
    assert abs(z.mean()) < 0.03
    assert abs(z.var() - 1.0) < 0.04


def test_decide_ncell_matches_reference_rule(orc):
    # DecideNumCell: floor(L * (1/cellSize)), < 4 in a direction -> no cell list
    assert orc.decide_ncell([16.796] * 3, 2.8) == ((5, 5, 5), True)
    assert orc.decide_ncell([40.0, 40.0, 160.0], 5.3) == ((7, 7, 30), True)
    assert orc.decide_ncell([10.0, 10.0, 10.0], 3.0)[1] is False


def test_bin_known_answers(orc):
    box = np.array([10.0, 10.0, 10.0], np.float32)
    nc = (4, 4, 4)
    pos = np.array([[0.0, 0.0, 0.0],      # cell 0
                    [9.9999995, 2.6, 5.1],  # x just below L
                    [-0.5, 10.5, 3.0],    # wraps: x -> 9.5 image -1, y -> 0.5 image +1
                    [2.5, 2.5, 2.5]],     # exactly on a cell edge -> cell (1,1,1)
                   np.float32)
    p, img, cell = orc.bin_f32(pos, box, nc)
    assert cell[0] == 0
    assert tuple(img[2]) == (-1, 1, 0)
    assert np.allclose(p[2], [9.5, 0.5, 3.0])
    assert cell[3] == 1 + 4 * (1 + 4 * 1)
    c1 = cell[1]
    assert c1 // 16 == 3 and (c1 // 4) % 4 == 1 and c1 % 4 == 2


def test_bin_wrap_fix_when_index_equals_ncell(orc):
    # x*sizei*NCell rounds up to NCell for the largest float below L: the
    # reference moves the atom by -L and bumps the image (NeighborList.cu:110-124)
    L = np.float32(7.0)
    box = np.array([L, L, L], np.float32)
    x = np.nextafter(L, np.float32(0))
    inv = np.float32(1) / L
    assert np.float32(np.float32(x * inv) * np.float32(4)) == np.float32(4)
    p, img, cell = orc.bin_f32(np.array([[x, 1.0, 1.0]], np.float32), box, (4, 4, 4))
    assert img[0, 0] == 1 and p[0, 0] < 0 and cell[0] // 16 == 0


def test_nlist_strict_boundary(orc):
    # a pair whose binary32 |d|^2 equals rlist^2 exactly is excluded (strict <)
    box = np.array([20.0, 20.0, 20.0], np.float32)
    pos = np.array([[5.0, 5.0, 5.0], [7.5, 5.0, 5.0], [5.0, 7.4999995, 5.0]], np.float32)
    rc = np.array([2.5, 2.5, 2.5], np.float32)
    counts, pairs = orc.nlist_allpair_f32(pos, rc, 0.0, box)
    assert counts.tolist() == [1, 0, 1]
    assert pairs.tolist() == [2, 0]


def test_nlist_min_image_across_boundary(orc):
    box = np.array([10.0, 10.0, 10.0], np.float32)
    pos = np.array([[0.2, 5.0, 5.0], [9.9, 5.0, 5.0]], np.float32)
    counts, pairs = orc.nlist_allpair_f32(pos, np.array([0.2, 0.2], np.float32), 0.15, box)
    assert counts.tolist() == [1, 1]


def test_cellshift_equals_allpair_away_from_ties(orc, mdf):
    s = mdf.systems.lj_fluid_fcc(cells=8, L=13.44)
    box = s.box.astype(np.float32)
    nc, ok = orc.decide_ncell(s.box, 2.8)
    assert ok
    p, _, cell = orc.bin_f32(s.pos, box, nc)
    c1, q1 = orc.nlist_cellshift_f32(p, cell, 2.8, box, nc)
    c2, q2 = orc.nlist_allpair_f32(p, np.full(len(p), 2.5, np.float32), 0.3, box)
    # both criteria may only differ on pairs within a few ulp of rlist
    assert abs(int(c1.sum()) - int(c2.sum())) <= 4
    assert c1.sum() > 50 * len(p)


def test_lj_oracle_two_body_and_newton(orc):
    box = np.array([30.0, 30.0, 30.0])
    pos = np.array([[1.0, 1.0, 1.0], [2.2, 1.0, 1.0]])
    F, st = orc.lj_allpair_f64(pos, np.array([2.5, 2.5]), box)
    r = 1.2
    fmag = 4 * (12 / r ** 13 - 6 / r ** 7)  # -dU/dr, repulsive positive
    assert np.allclose(F[0], [-fmag, 0, 0], rtol=1e-14)
    assert np.allclose(F[1], [fmag, 0, 0], rtol=1e-14)
    assert np.isclose(st[0], 4 * (r ** -12 - r ** -6), rtol=1e-14)
    # asymmetric adaptive cutoff: atom 0 sees 1, atom 1 (rc 1.0) does not see 0
    F, _ = orc.lj_allpair_f64(pos, np.array([2.5, 1.0]), box)
    assert np.allclose(F[1], 0) and not np.allclose(F[0], 0)


def test_assign_rcut_oracle(orc):
    box = np.array([10.0, 10.0, 30.0], np.float32)
    lat = np.arange(3 * 3 * 5, dtype=np.float32).reshape(3, 3, 5) + 1
    pos = np.array([[0.1, 0.1, 0.1], [9.99, 9.99, 29.9], [-0.1, 5.0, 15.0]], np.float32)
    rc = orc.assign_rcut_f32(pos, box, lat)
    assert rc[0] == lat[0, 0, 0] and rc[1] == lat[2, 2, 4] and rc[2] == lat[2, 1, 2]


def test_generators(mdf):
    s = mdf.systems.lj_fluid_fcc()
    assert s.pos.shape == (4000, 3)
    assert np.isclose(4000 / s.box.prod(), 0.8442, atol=2e-4)
    assert np.allclose(s.vel.mean(0), 0, atol=1e-12)
    s2 = mdf.systems.lj_fluid_fcc()
    assert np.array_equal(s.pos, s2.pos)
    c = mdf.systems.charged_fluid(n=2000, L=14.0)
    assert c.charge.sum() == 0 and set(np.unique(c.charge)) == {-1.0, 1.0}
    d = c.pos[:, None, :] - c.pos[None, :, :]
    d -= np.round(d / 14.0) * 14.0
    r2 = (d ** 2).sum(-1) + np.eye(2000) * 1e9
    assert r2.min() >= 0.8 ** 2 - 1e-12


def test_slab_generator_counts(mdf):
    s = mdf.systems.lj_slab(n=8192, box=(20.0, 20.0, 80.0))
    hw = s.meta["liquid_half_width"]
    inside = np.abs(s.pos[:, 2] - 40.0) < hw
    assert inside.sum() == s.meta["n_liquid"]
    rho_l = inside.sum() / (400 * 2 * hw)
    rho_v = (~inside).sum() / (400 * (80 - 2 * hw))
    assert abs(rho_l - 0.78) < 0.01 and abs(rho_v - 0.02) < 0.005


def test_host_side_errors_without_gpu(mdf):
    # bad arguments are rejected on the host before any device call
    with pytest.raises(mdf.MDExcptBadArgument):
        mdf.MDSystem(np.full((4, 3), np.nan), [10, 10, 10])
    with pytest.raises(mdf.MDExcptBadArgument):
        mdf.MDSystem(np.zeros((4, 3)), [10, -1, 10])


def test_oracle_md_runs_and_thermostats(orc, mdf):
    s = mdf.systems.lj_fluid_fcc(cells=4, L=6.72)
    out = orc.md_langevin_run(s.pos, s.vel, s.box, 200, dt=0.005, temperature=1.0, gamma_t=1.0,
                              skin=0.3, rcut=np.full(s.n, 2.5, np.float32), seed=3)
    assert out["status"] == 0
    K = out["stats"][4:7].sum()
    T = 2 * K / (3 * s.n)
    assert 0.7 < T < 1.3
    assert out["rebuilds"] >= 1
