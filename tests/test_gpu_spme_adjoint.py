"""GPU tests of the SPME adjoint (md_spme_energy_grad) and its
torch.autograd.Function: gradients of the reciprocal energy with respect to
charges, positions, the splitting beta and the influence function, against
FP64 finite differences, the analytic-differentiation forces of the forward
path and of the oracle, and the quadratic-form identities
E = 1/2 sum_i q_i dE/dq_i and E = sum_m psi(m) dE/dpsi(m)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.fixture(scope="module")
def small():
    rng = np.random.default_rng(5)
    n, L = 300, 9.0
    pos = rng.uniform(0, L, (n, 3))
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0) * rng.uniform(0.5, 1.5, n)
    return pos, q, np.array([L, L, L])


def make(mdf, pos, q, box, prec=1, method="ik", K=(16, 16, 32), order=6, beta=1.3):
    sys = mdf.MDSystem(pos, box, charge=q, precision=prec)
    return sys, mdf.SPME(sys, K, order, beta, method)


def test_energy_and_position_gradient(mdf, orc, small):
    pos, q, box = small
    sys, sp = make(mdf, pos, q, box)
    out = sp.energy_grad(dpsi=True)
    # energy equals the forward path's reciprocal energy
    eng = mdf.InteractionEngine(sys)
    eng.clearInteraction()
    sys.clear_stats()
    sp.apply()
    assert abs(out["energy"] - sys.stats()[mdf.STAT_ELEC_REC]) < 1e-12 * abs(out["energy"])
    # dE/dr is minus the analytic-differentiation force, forward path and oracle
    sys2, sp2 = make(mdf, pos, q, box, method="analytic")
    eng2 = mdf.InteractionEngine(sys2)
    eng2.clearInteraction()
    sp2.apply()
    assert rel(out["dE_dr"], -sys2.forces()) < 1e-12
    _, Fo = orc.spme_rec(pos, q, box, (16, 16, 32), 6, 1.3, 1)
    assert rel(out["dE_dr"], -Fo) < 1e-10
    Eo, _ = orc.spme_rec(pos, q, box, (16, 16, 32), 6, 1.3, 0)
    assert abs(out["energy"] - Eo) < 1e-10 * abs(Eo)
    # quadratic forms: E = 1/2 q . dE/dq, and E is linear in psi
    assert abs(0.5 * q @ out["dE_dq"] - out["energy"]) < 1e-12 * abs(out["energy"])
    assert abs((sp.influence() * out["dE_dpsi"]).sum() - out["energy"]) < 1e-12 * abs(out["energy"])


def test_finite_differences_fp64(mdf, small):
    pos, q, box = small
    sys, sp = make(mdf, pos, q, box)
    out = sp.energy_grad()
    E = lambda: sp.energy_grad(dq=False, dr=False)["energy"]  # noqa: E731
    h = 1e-6
    for i in (0, 17, 123, 299):
        qq = q.copy()
        qq[i] += h
        sys.set_charges(qq)
        ep = E()
        qq[i] -= 2 * h
        sys.set_charges(qq)
        em = E()
        sys.set_charges(q)
        fd = (ep - em) / (2 * h)
        assert abs(fd - out["dE_dq"][i]) <= 1e-6 * abs(out["dE_dq"][i]) + 1e-9
        for d in range(3):
            pp = pos.copy()
            pp[i, d] += h
            sys.set_positions(pp)
            ep = E()
            pp[i, d] -= 2 * h
            sys.set_positions(pp)
            em = E()
            sys.set_positions(pos)
            fd = (ep - em) / (2 * h)
            assert abs(fd - out["dE_dr"][i, d]) <= 1e-6 * np.abs(out["dE_dr"][i]).max() + 1e-9
    # splitting parameter
    hb = 1e-6
    e_p = make(mdf, pos, q, box, beta=1.3 + hb)[1].energy_grad(dq=False, dr=False)["energy"]
    e_m = make(mdf, pos, q, box, beta=1.3 - hb)[1].energy_grad(dq=False, dr=False)["energy"]
    assert abs((e_p - e_m) / (2 * hb) - out["dE_dbeta"]) <= 1e-6 * abs(out["dE_dbeta"])


def test_mixed_precision_adjoint_tracks_fp64(mdf, small):
    pos, q, box = small
    ref = make(mdf, pos, q, box, prec=1)[1].energy_grad()
    mix = make(mdf, pos, q, box, prec=0)[1].energy_grad()
    assert abs(mix["energy"] - ref["energy"]) < 1e-5 * abs(ref["energy"])
    assert rel(mix["dE_dq"], ref["dE_dq"]) < 1e-5
    assert rel(mix["dE_dr"], ref["dE_dr"]) < 1e-4


def test_autograd_function(mdf, small):
    import torch
    from mdforce.optibasis import spme_energy
    pos, q, box = small
    sys, sp = make(mdf, pos, q, box)
    ref = sp.energy_grad()
    for recompute in (False, True):
        qt = torch.tensor(q, dtype=torch.float64, requires_grad=True)
        rt = torch.tensor(pos, dtype=torch.float64, requires_grad=True)
        E = spme_energy(qt, rt, sp, recompute=recompute)
        (3.0 * E).backward()
        assert abs(E.item() - ref["energy"]) < 1e-13 * abs(ref["energy"])
        assert rel(qt.grad.numpy(), 3.0 * ref["dE_dq"]) < 1e-13
        assert rel(rt.grad.numpy(), 3.0 * ref["dE_dr"]) < 1e-13


def test_autograd_function_device_tensors(mdf, small):
    """CUDA tensors go to the system as raw device pointers and the gradients
    come back in device memory (md_system_set_device_view,
    md_spme_energy_grad_device): the same values as the host path."""
    import torch
    from mdforce.optibasis import spme_energy
    pos, q, box = small
    sys, sp = make(mdf, pos, q, box)
    ref = sp.energy_grad()
    for recompute in (False, True):
        qt = torch.tensor(q, dtype=torch.float64, device="cuda", requires_grad=True)
        rt = torch.tensor(pos, dtype=torch.float64, device="cuda", requires_grad=True)
        E = spme_energy(qt, rt, sp, recompute=recompute)
        assert E.is_cuda
        (3.0 * E).backward()
        assert abs(E.item() - ref["energy"]) < 1e-13 * abs(ref["energy"])
        assert rel(qt.grad.cpu().numpy(), 3.0 * ref["dE_dq"]) < 1e-13
        assert rel(rt.grad.cpu().numpy(), 3.0 * ref["dE_dr"]) < 1e-13
    # moved positions reach the system through the view
    rt = torch.tensor(pos + 0.01, dtype=torch.float64, device="cuda")
    E2 = spme_energy(torch.tensor(q, dtype=torch.float64, device="cuda"), rt, sp)
    sys.set_positions(pos + 0.01)
    assert abs(E2.item() - sp.energy_grad(dq=False, dr=False)["energy"]) < 1e-13 * abs(E2.item())


def test_autograd_gradcheck(mdf):
    import torch
    from mdforce.optibasis import spme_energy
    rng = np.random.default_rng(9)
    n, L = 24, 6.0
    pos = rng.uniform(0, L, (n, 3))
    q = rng.uniform(-1, 1, n)
    sys, sp = make(mdf, pos, q, np.array([L, L, L]), K=(16, 16, 16), order=4, beta=1.1)
    qt = torch.tensor(q, dtype=torch.float64, requires_grad=True)
    rt = torch.tensor(pos, dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(lambda a, b: spme_energy(a, b, sp), (qt, rt), eps=1e-6, atol=1e-7, rtol=1e-6)


def test_charged_fluid_identities(mdf):
    """20736 unit charges, 30^3 box, 64^3 mesh, order 6, beta 0.95 (the
    charged-fluid system): size-independent checks at full size."""
    s = mdf.systems.charged_fluid()
    sys, sp = make(mdf, s.pos, s.charge, s.box, prec=1, K=(64, 64, 64), order=6, beta=0.95)
    out = sp.energy_grad()
    assert abs(0.5 * s.charge @ out["dE_dq"] - out["energy"]) < 1e-11 * abs(out["energy"])
    sys2, sp2 = make(mdf, s.pos, s.charge, s.box, prec=1, method="analytic", K=(64, 64, 64), order=6, beta=0.95)
    eng = mdf.InteractionEngine(sys2)
    eng.clearInteraction()
    sp2.apply()
    assert rel(out["dE_dr"], -sys2.forces()) < 1e-11
    # central differences on a few atoms; the energy sums 1.4e5 modes, so its
    # rounding (~1e-11 absolute) needs a step of 1e-4 (truncation ~1e-9 for the
    # order-6 spline) rather than the 1e-6 used on the small system
    E = lambda: sp.energy_grad(dq=False, dr=False)["energy"]  # noqa: E731
    h = 1e-4
    for i in (5, 10000):
        pp = s.pos.copy()
        pp[i, 2] += h
        sys.set_positions(pp)
        ep = E()
        pp[i, 2] -= 2 * h
        sys.set_positions(pp)
        em = E()
        sys.set_positions(s.pos)
        assert abs((ep - em) / (2 * h) - out["dE_dr"][i, 2]) <= 1e-6 * np.abs(out["dE_dr"][i]).max() + 1e-8
