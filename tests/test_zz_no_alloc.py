"""GPU test of md_error_estimate_spme_ik_noalloc, the allocation-free variant of
the ik-SPME interpolation estimate: called through the C ABI twice in a row, it
must agree with md_error_estimate_spme_ik on the same system, and meshes beyond
its fixed scratch must be rejected with MD_ERR_BADARG. The file name keeps it
last in collection so that it also runs after every other GPU test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _estimate(lib, fn, sys, K, order, beta):
    KK = (C.c_int * 3)(*K)
    e = C.c_double()
    rc = getattr(lib, fn)(sys.h, KK, int(order), float(beta), C.byref(e))
    return rc, e.value


@pytest.mark.parametrize("prec", [0, 1])
def test_noalloc_matches_allocating_estimate(mdf, prec):
    from mdforce._lib import lib
    rng = np.random.default_rng(3)
    n, L = 400, 10.0
    pos = rng.uniform(0, L, (n, 3))
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    sys = mdf.MDSystem(pos, np.array([L, L, L]), charge=q, precision=prec)
    for K, order, beta in (((16, 16, 32), 6, 1.3), ((32, 32, 32), 4, 1.1), ((160, 160, 160), 6, 2.0)):
        rc, ref = _estimate(lib, "md_error_estimate_spme_ik", sys, K, order, beta)
        assert rc == 0
        for _ in range(2):  # two calls in a row reuse the same scratch
            rc, e = _estimate(lib, "md_error_estimate_spme_ik_noalloc", sys, K, order, beta)
            assert rc == 0, lib.md_last_error_message()
            assert abs(e - ref) <= 1e-13 * ref, (K, e, ref)


def test_noalloc_rejects_meshes_beyond_scratch(mdf):
    from mdforce._lib import lib
    rng = np.random.default_rng(4)
    pos = rng.uniform(0, 8.0, (64, 3))
    q = np.where(np.arange(64) % 2 == 0, 1.0, -1.0)
    sys = mdf.MDSystem(pos, np.array([8.0, 8.0, 8.0]), charge=q, precision=1)
    rc, _ = _estimate(lib, "md_error_estimate_spme_ik_noalloc", sys, (256, 256, 256), 6, 1.0)
    assert rc == mdf.MD_ERR_BADARG
    msg = lib.md_last_error_message()
    msg = msg.decode() if isinstance(msg, bytes) else str(msg)
    assert "4194304" in msg
    # the system stays usable after the rejection
    rc, e = _estimate(lib, "md_error_estimate_spme_ik_noalloc", sys, (16, 16, 16), 6, 1.0)
    assert rc == 0 and e > 0
