"""The oracle's non-bonded pair kinds (oracle_md.c nb_pair) against the reference
engine's own pair functions (include/NonBondedInteraction.h, the nbForcePoten
dispatch) compiled as host code in oracle/_ref: bit-equal in binary32."""
import numpy as np
import pytest

KINDS = [(1, (1.2, 0.9, 0.05, 3.0)), (5, (1.1, 1.0, 0.1, 2.2)), (3, (1.0, 0.95, 1.6)), (3, (1.0, 0.95, 0.0)),
         (2, (1.2, 0.9, 0.05, 2.5, 50.0)), (6, (1.1, 1.0, 0.1, 2.2, 40.0)), (4, (1.0, 0.95, 1.6, 30.0))]


@pytest.mark.parametrize("kind,u", KINDS)
def test_pairs_equal_the_reference_header(orc, kind, u):
    if not orc.ref_available("libref_nb.so"):
        pytest.skip("reference non-bonded header not built (needs the reference tree at build time)")
    rng = np.random.default_rng(kind)
    for _ in range(1000):
        d = rng.normal(size=3)
        d *= rng.uniform(0.6, 3.0) / np.linalg.norm(d)  # the capped kinds' cores included
        f, e = orc.nb_pair(kind, u, 0, d)
        rf, re = orc.ref_nb_pair(kind, u, d)
        assert np.array_equal(f, rf) and e == re


@pytest.mark.parametrize("kind,u", KINDS)
def test_fp64_pairs_track_binary32(orc, kind, u):
    rng = np.random.default_rng(10 + kind)
    for _ in range(300):
        d = rng.normal(size=3)
        d *= rng.uniform(0.9, 2.9) / np.linalg.norm(d)
        a, ea = orc.nb_pair(kind, u, 0, d)
        b, eb = orc.nb_pair(kind, u, 1, d)
        assert np.abs(a - b).max() <= 1e-4 * max(np.abs(b).max(), 1.0)
        assert abs(ea - eb) <= 1e-4 * max(abs(eb), 1.0)
