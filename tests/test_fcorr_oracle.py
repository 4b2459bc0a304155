"""CPU tests of the long-range force-correction (LFC) oracle: the field of
ForceCorr::makeS2k + calError (FCR = shortRange.inhomo/template/tools/
simulation.fcorr, FCR/src/ForceCorr.cu:150-262) restated in oracle.fcorr_field
against the reference's own ForceCorr compiled in oracle/_ref, and the
binary32 binning of AssignForceCorr::assign."""
import numpy as np
import pytest


def slab_profile(n, L, half, seed=0):
    z = (np.arange(n[2]) + 0.5) * L / n[2]
    rho = np.where(np.abs(z - L / 2) < half, 0.78, 0.02)
    rho = np.ascontiguousarray(np.broadcast_to(rho, n), np.float64)
    return rho * (1 + 0.05 * np.random.default_rng(seed).standard_normal(n))


@pytest.mark.parametrize("rc", [3.5, 5.0])
def test_fcorr_oracle_matches_reference_build(orc, rc):
    if not orc.ref_available("libref_fcorr.so"):
        pytest.skip("reference ForceCorr not built (needs the reference tree at build time)")
    box = [12.0, 12.0, 40.0]
    n = orc.dp_bins(box, 1.6)
    rho = slab_profile(n, box[2], 8.0)
    a = orc.fcorr_field(box, n, rc, rho)
    b = orc.ref_fcorr(box, n, rc, rho)
    scale = np.abs(b.real).max()
    assert scale > 0
    assert np.abs(a.real - b.real).max() < 1e-12 * scale
    assert np.abs(a.imag - b.imag).max() < 1e-12 * scale


def test_fcorr_field_properties(orc):
    """A homogeneous profile has no correction force; a slab's points along z
    (toward the liquid), antisymmetric about the slab centre, with no x or y
    component."""
    box = [10.0, 10.0, 40.0]
    n = orc.dp_bins(box, 2.0)
    f = orc.fcorr_field(box, n, 3.0, np.full(n, 0.5))
    assert np.abs(f).max() < 1e-12
    z = (np.arange(n[2]) + 0.5) * box[2] / n[2]
    rho = np.ascontiguousarray(np.broadcast_to(np.where(np.abs(z - 20.0) < 8.0, 0.8, 0.0), n), np.float64)
    f = orc.fcorr_field(box, n, 3.0, rho).real
    assert np.abs(f[0]).max() < 1e-12 and np.abs(f[1]).max() < 1e-12
    fz = f[2][0, 0]
    assert np.abs(fz + fz[::-1]).max() < 1e-10 * np.abs(fz).max()


def test_fcorr_assign_binning(orc):
    box = np.array([10.0, 10.0, 40.0])
    n = (5, 5, 21)
    field = np.arange(3 * np.prod(n), dtype=np.float64).reshape((3,) + n)
    pos = np.array([[0.0, 0.0, 0.0], [9.999, 5.0, 39.99], [-0.5, 10.2, 20.0], [2.0, 4.0, 1.905]])
    v = orc.fcorr_assign(pos, box, n, field)
    # wrapped once, then int((x * n) / L) in binary32
    exp_idx = [(0, 0, 0), (4, 2, 20), (4, 0, 10), (1, 2, 1)]
    for k, (ix, iy, iz) in enumerate(exp_idx):
        assert tuple(v[k]) == tuple(field[:, ix, iy, iz]), k
