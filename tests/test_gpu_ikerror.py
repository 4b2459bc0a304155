"""GPU tests of the optiBasis error functional (md_ikerr_*) through the C
ABI: values and basis gradients against the reference's own Python results
(tests/golden/ikerror_cases.json), hats and axis weights against the oracle,
the batched evaluation of 8 perturbed candidates on the charged-fluid mesh
(64^3, 16 Hermite bins, box 30, beta 0.95) against the oracle, and the
torch.autograd path against finite differences."""
import json
import os

import numpy as np
import pytest

from oracle.ikerror import IkErrorOracle

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ikerror_cases.json")


def cases():
    with open(GOLDEN) as f:
        return json.load(f)["cases"]


def gpu_functional(mdf, c):
    cls = mdf.optibasis.HermiteLossFunc_Bound0 if c["bound0"] else mdf.optibasis.HermiteLossFunc
    return cls(c["CC"], c["nbin"], c["beta"], c["KK"], c["q2"], c["natoms"], c["L"], l_cut=c["l_cut"])


@pytest.mark.parametrize("name", [c["name"] for c in cases()])
def test_matches_reference_values_and_gradients(mdf, name):
    c = next(c for c in cases() if c["name"] == name)
    f = gpu_functional(mdf, c)
    for e in c["evals"]:
        assert abs(f.value(e["vv"]) - e["value"]) < 1e-12 * e["value"]
        d, dr = f.deriv(e["vv"]), np.array(e["deriv"])
        assert np.abs(d - dr).max() < 1e-11 * np.abs(dr).max()
    # the hat of the current basis along axis 0, as the reference's buffer
    h0, hb = f.hats(0)
    hat = h0 + np.array(c["evals"][1]["vv"]) @ hb
    assert np.abs(hat - np.array(c["hat_axis0_last"])).max() < 1e-15


@pytest.fixture(scope="module")
def charged_mesh(mdf):
    # the charged-fluid system: 20736 unit charges, box 30, beta 0.95, mesh 64^3;
    # 16 Hermite bins on [0, 2] starting from the order-4 B-spline
    p = dict(CC=2, nbin=16, beta=0.95, KK=[64, 64, 64], L=[30.0, 30.0, 30.0], q2=20736.0, natoms=20736.0,
             l_cut=10)
    f = mdf.optibasis.HermiteLossFunc(p["CC"], p["nbin"], p["beta"], p["KK"], p["q2"], p["natoms"], p["L"],
                                      l_cut=p["l_cut"])
    o = IkErrorOracle(p["CC"], p["nbin"], p["beta"], p["KK"], p["L"], p["q2"], p["natoms"], p["l_cut"], False)
    v0 = mdf.optibasis.bspline_initial_basis(p["CC"], p["nbin"], 4)
    rng = np.random.default_rng(11)
    V = v0[None, :] + rng.normal(0.0, 0.1, (8, v0.size))
    V[0] = v0
    return f, o, V


def test_hats_and_weights_match_oracle(charged_mesh):
    f, o, _ = charged_mesh
    for d in range(3):
        h0, hb = f.hats(d)
        oh0, ohb = o.hats[d]
        assert np.abs(h0 - oh0).max() < 1e-15
        assert np.abs(hb - ohb).max() < 1e-15
        W = f.weights(d)
        assert np.abs(W - o.W[d]).max() < 1e-12 * np.abs(o.W[d]).max()


def test_batch_of_candidates_matches_oracle(charged_mesh):
    f, o, V = charged_mesh
    val, g = f.evaluate(V)
    for c in range(V.shape[0]):
        assert abs(val[c] - o.value(V[c])) < 1e-11 * val[c]
        og = o.deriv(V[c])
        assert np.abs(g[c] - og).max() < 1e-10 * np.abs(og).max()


def test_autograd_on_device_against_finite_differences(charged_mesh):
    import torch
    from mdforce.optibasis import ik_error_loss
    f, _, V = charged_mesh
    x = torch.tensor(V[:4], dtype=torch.float64, device="cuda", requires_grad=True)
    y = ik_error_loss(x, f)
    w = torch.tensor([1.0, -0.5, 0.25, 2.0], dtype=torch.float64, device="cuda")
    (y * w).sum().backward()
    g = x.grad.cpu().numpy()
    val, gh = f.evaluate(V[:4])
    assert np.allclose(y.detach().cpu().numpy(), val, rtol=1e-14, atol=0)
    assert np.allclose(g, gh * w.cpu().numpy()[:, None], rtol=1e-14, atol=0)
    # five-point differences of the device values (see the oracle test for the step)
    h = 1e-6
    for b in (0, 7, 20, 31):
        e = np.zeros(V.shape[1])
        e[b] = h
        fv = [f.value(V[1] + k * e) for k in (2, 1, -1, -2)]
        fd = (-fv[0] + 8 * fv[1] - 8 * fv[2] + fv[3]) / (12 * h)
        assert abs(fd - gh[1, b]) < 1e-6 * np.abs(gh[1]).max()


def test_bad_arguments_are_rejected(mdf):
    with pytest.raises(mdf.MDException):
        mdf.optibasis.HermiteLossFunc(2, 10, 1.0, [16, 16, 16], 1.0, 1.0, [3.0, 3.0, 3.0], l_cut=500)
    f = mdf.optibasis.HermiteLossFunc(2, 4, 3.0, [8, 8, 8], 1.0, 3.0, [2.0, 2.0, 2.0], l_cut=2)
    with pytest.raises(ValueError):
        f.evaluate(np.zeros((2, 5)))
