"""The oracle's bonded terms (oracle_bonded.c) against the reference engine's own
force functions (include/BondInteraction.h, include/AngleInteraction.h) compiled
as host code in oracle/_ref: bit-equal in binary32 for every term type."""
import numpy as np
import pytest

TERMS = [(10000, (30.0, 1.0)), (10001, (30.0, 1.5)), (10002, (20.0, 0.8, 1.0)), (20000, (5.0, 1.9)),
         (20001, (3.0,))]


@pytest.mark.parametrize("ftype,u", TERMS)
def test_terms_equal_the_reference_headers(orc, ftype, u):
    if not orc.ref_available("libref_bonded.so"):
        pytest.skip("reference bonded headers not built (needs the reference tree at build time)")
    rng = np.random.default_rng(ftype)
    for _ in range(500):
        d0 = rng.normal(0, 0.6, 3)
        d1 = rng.normal(0, 0.6, 3)
        if ftype < 20000:
            n = np.linalg.norm(d0)
            if n > 1.3:
                d0 *= 1.2 / n
            f, e = orc.bond_term(ftype, u, 0, d0)
            rf, re = orc.ref_bonded_term(ftype, u, d0)
            assert np.array_equal(f, rf) and e == re
        else:
            f0, f1, e = orc.angle_term(ftype, u, 0, d0, d1)
            r0, r1, re = orc.ref_bonded_term(ftype, u, d0, d1)
            assert np.array_equal(f0, r0) and np.array_equal(f1, r1) and e == re


def test_fp64_terms_track_binary32(orc):
    """The binary64 evaluation of each term agrees with binary32 to its rounding."""
    rng = np.random.default_rng(1)
    for ftype, u in TERMS:
        for _ in range(200):
            d0 = rng.normal(0, 0.5, 3)
            d1 = rng.normal(0, 0.5, 3)
            if ftype < 20000:
                d0 *= min(1.0, 1.1 / np.linalg.norm(d0))
                a, ea = orc.bond_term(ftype, u, 0, d0)
                b, eb = orc.bond_term(ftype, u, 1, d0)
                assert np.abs(a - b).max() <= 1e-4 * max(np.abs(b).max(), 1.0)
            else:
                a0, a1, ea = orc.angle_term(ftype, u, 0, d0, d1)
                b0, b1, eb = orc.angle_term(ftype, u, 1, d0, d1)
                assert np.abs(a0 - b0).max() <= 1e-3 * max(np.abs(b0).max(), 1.0)
            assert abs(ea - eb) <= 1e-4 * max(abs(eb), 1.0)


def test_gathered_forces_sum_to_zero(orc):
    """Per-atom gather over a small chain: the bonded forces balance."""
    pos = np.array([[1.0, 1.0, 1.0], [1.9, 1.2, 1.0], [2.5, 1.9, 1.3], [3.4, 2.0, 1.9]])
    box = np.full(3, 10.0)
    F, st = orc.bonded_apply(pos, box, 1, [[0, 1], [1, 2], [2, 3]], [10000, 10001, 10002],
                             [[50, 1.0, 0], [30, 1.5, 0], [20, 0.8, 0.95]], [[0, 1, 2], [1, 2, 3]],
                             [20000, 20001], [[5.0, 1.9, 0], [3.0, 0, 0]])
    assert np.abs(F.sum(axis=0)).max() < 1e-12 * np.abs(F).max()
    assert st[0] > 0
