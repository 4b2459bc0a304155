"""optiBasis side: the ik-SPME force-error functional of a piecewise cubic
Hermite interpolation basis and its gradient, evaluated on the GPU through
the C ABI (md_ikerr_*), with a torch.autograd.Function for gradient-based
basis optimisation.

Mirrors optiBasis/IkError.py: HermiteLossFunc and HermiteLossFunc_Bound0
(:166-260) keep their constructor arguments and their value(vv) / deriv(vv)
methods, so optiBasis/compute_basis.py can hand them to
scipy.optimize.minimize unchanged.  The coefficient vector is
[v_1..v_n, d_1..d_n] (optiBasis/basis_common.py unpack_v_d).
"""
import ctypes as C

import numpy as np

from ._lib import lib
from .core import check

CONVERSION = 138.93545756169981341199  # optiBasis/IkError.py:25

_P = C.POINTER(C.c_double)


def _box_of(region):
    """Box lengths from a 3-vector or from an object with a diagonal 3x3 `mat`
    (optiBasis/Region.py)."""
    if hasattr(region, "mat"):
        m = np.asarray(region.mat, dtype=float)
        if np.abs(m - np.diag(np.diag(m))).max() > 0:
            raise ValueError("only rectangular regions are supported")
        return np.diag(m).copy()
    b = np.asarray(region, dtype=float).reshape(-1)
    return np.repeat(b, 3) if b.size == 1 else b


class IkErrorGPU:
    """Device-resident functional for one (basis layout, mesh, box, beta).

    value(vv), deriv(vv) take one coefficient vector; evaluate(V) takes a
    batch [C, n] and returns (values [C], grads [C, n])."""

    def __init__(self, CC, nbin, beta, KK, q2, natoms, region, l_cut=10, bound0=False, over_smpl=0, device=0):
        K = [int(k) for k in (KK if np.ndim(KK) else [KK] * 3)]
        L = _box_of(region)
        h = C.c_void_p()
        check(lib.md_ikerr_create(C.byref(h), (C.c_int * 3)(*K), (C.c_double * 3)(*L), float(beta), float(CC),
                                  int(nbin), int(l_cut), 1 if bound0 else 0, int(over_smpl), float(q2),
                                  float(natoms), int(device)), "md_ikerr_create")
        self.h = h
        self.K, self.L, self.l_cut = K, L, int(l_cut)
        n = C.c_int()
        check(lib.md_ikerr_num_coeffs(self.h, C.byref(n)), "md_ikerr_num_coeffs")
        self.ncoef = n.value

    def __del__(self):
        if getattr(self, "h", None):
            lib.md_ikerr_destroy(self.h)
            self.h = None

    def evaluate(self, V, grads=True):
        V = np.ascontiguousarray(np.atleast_2d(np.asarray(V, dtype=np.float64)))
        if V.shape[1] != self.ncoef:
            raise ValueError(f"expected {self.ncoef} coefficients, got {V.shape[1]}")
        nc = V.shape[0]
        val = np.zeros(nc)
        g = np.zeros((nc, self.ncoef)) if grads else None
        check(lib.md_ikerr_evaluate(self.h, nc, V.ctypes.data_as(_P), val.ctypes.data_as(_P),
                                    g.ctypes.data_as(_P) if grads else None), "md_ikerr_evaluate")
        return val, g

    def evaluate_device(self, d_coeffs, d_values, d_grads, nc, stream=None):
        """Raw device pointers (ints), asynchronous on `stream` (an int handle)."""
        check(lib.md_ikerr_evaluate_device(self.h, int(nc), C.c_void_p(d_coeffs), C.c_void_p(d_values),
                                           C.c_void_p(d_grads) if d_grads else None,
                                           C.c_void_p(stream) if stream else None), "md_ikerr_evaluate_device")

    def value(self, vv):
        return float(self.evaluate(vv, grads=False)[0][0])

    def deriv(self, vv):
        return self.evaluate(vv, grads=True)[1][0]

    def hats(self, d=0):
        kmax = self.K[d] // 2 + self.l_cut * self.K[d]
        h0 = np.zeros(kmax + 1)
        hb = np.zeros((self.ncoef, kmax + 1))
        check(lib.md_ikerr_get_hats(self.h, int(d), h0.ctypes.data_as(_P), hb.ctypes.data_as(_P)), "hats")
        return h0, hb

    def weights(self, d=0):
        W = np.zeros(self.K[d] + 1)
        check(lib.md_ikerr_get_weights(self.h, int(d), W.ctypes.data_as(_P)), "weights")
        return W


class HermiteLossFunc(IkErrorGPU):
    """optiBasis/IkError.py:166-212: basis with free value and slope at CC
    (2 nbin coefficients)."""

    def __init__(self, CC, nbin, beta, KK, q2, natoms, region, l_cut=10, device=0):
        super().__init__(CC, nbin, beta, KK, q2, natoms, region, l_cut=l_cut, bound0=False, device=device)


class HermiteLossFunc_Bound0(IkErrorGPU):
    """optiBasis/IkError.py:214-260: basis vanishing at CC (2 nbin - 2
    coefficients)."""

    def __init__(self, CC, nbin, beta, KK, q2, natoms, region, l_cut=10, device=0):
        super().__init__(CC, nbin, beta, KK, q2, natoms, region, l_cut=l_cut, bound0=True, device=device)


def _torch():
    import torch
    return torch


def ik_error_loss(coeffs, functional):
    """Force-error estimates of a batch of candidate bases, differentiable
    with respect to the coefficients: coeffs is a float64 tensor [C, n] (or
    [n]) on the CPU or on the functional's GPU; returns [C] (or a scalar)."""
    torch = _torch()

    class _IkErrorLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x):
            squeeze = x.dim() == 1
            xb = x.detach().reshape(-1, functional.ncoef).to(torch.float64).contiguous()
            nc = xb.shape[0]
            if xb.is_cuda:
                val = torch.empty(nc, dtype=torch.float64, device=xb.device)
                grad = torch.empty(nc, functional.ncoef, dtype=torch.float64, device=xb.device)
                functional.evaluate_device(xb.data_ptr(), val.data_ptr(), grad.data_ptr(), nc,
                                           torch.cuda.current_stream(xb.device).cuda_stream)
            else:
                v, g = functional.evaluate(xb.numpy(), grads=True)
                val, grad = torch.from_numpy(v), torch.from_numpy(g)
            ctx.save_for_backward(grad)
            ctx.squeeze = squeeze
            return val[0] if squeeze else val

        @staticmethod
        def backward(ctx, gout):
            (grad,) = ctx.saved_tensors
            if ctx.squeeze:
                return (gout * grad[0]).to(gout.dtype)
            return (gout.reshape(-1, 1) * grad).to(gout.dtype)

    return _IkErrorLoss.apply(coeffs)


def spme_energy(q, r, spme, recompute=False):
    """Reciprocal SPME energy of charges q [N] at positions r [N, 3] (float64
    tensors), differentiable in both through the hand-written adjoint
    (md_spme_energy_grad).  The system of `spme` takes q and r on every call:
    CUDA tensors are handed over as raw device pointers on torch's current
    stream (md_system_set_device_view, md_spme_energy_grad_device: no host
    copy, no wait); CPU tensors go through host arrays.  With recompute=True
    the forward keeps nothing but the inputs and the backward recomputes
    spread, transforms and gather (memory-lean); by default the gradient comes
    with the forward pass and is kept for the backward."""
    torch = _torch()
    sys_ = spme.sys

    def run(qq, rr, grads):
        if qq.is_cuda:
            qd = qq.detach().to(torch.float64).contiguous()
            rd = rr.detach().to(torch.float64).contiguous()
            sys_.set_stream(torch.cuda.current_stream(qd.device).cuda_stream)
            sys_.set_device_view(rd.data_ptr(), qd.data_ptr())
            e = torch.empty(2, dtype=torch.float64, device=qd.device)
            gq = torch.empty_like(qd) if grads else None
            gr = torch.empty_like(rd) if grads else None
            spme.energy_grad_device(e.data_ptr(), gq.data_ptr() if grads else None,
                                    gr.data_ptr() if grads else None, e[1:].data_ptr())
            return e[0], gq, gr
        sys_.set_charges(qq.detach().numpy())
        sys_.set_positions(rr.detach().numpy())
        out = spme.energy_grad(dq=grads, dr=grads)
        e = torch.tensor(out["energy"], dtype=torch.float64)
        if not grads:
            return e, None, None
        return e, torch.from_numpy(out["dE_dq"]), torch.from_numpy(out["dE_dr"])

    class _SPMEEnergy(torch.autograd.Function):
        @staticmethod
        def forward(ctx, qq, rr):
            e, gq, gr = run(qq, rr, not recompute)
            if recompute:
                ctx.save_for_backward(qq, rr)
            else:
                ctx.save_for_backward(gq, gr)
            return e

        @staticmethod
        def backward(ctx, g):
            a, b = ctx.saved_tensors
            if recompute:
                _, gq, gr = run(a, b, True)
            else:
                gq, gr = a, b
            return (g * gq).to(gq.dtype), (g * gr).to(gr.dtype)

    return _SPMEEnergy.apply(q, r)


class HermiteSPME:
    """ik-SPME whose interpolation basis is the piecewise cubic Hermite basis of
    optiBasis (coefficients [v_1..v_n, d_1..d_n] as HermiteLossFunc(_Bound0)),
    for natoms charges on mesh K in box L with splitting beta, on the GPU in
    FP64 (md_hspme_*).  Inputs and outputs are CUDA float64 tensors handed over
    as raw device pointers on torch's current stream."""

    def __init__(self, natoms, K, L, beta, CC, nbin, bound0=False, device=0):
        K = [int(k) for k in (K if np.ndim(K) else [K] * 3)]
        L = _box_of(L)
        h = C.c_void_p()
        check(lib.md_hspme_create(C.byref(h), int(natoms), (C.c_int * 3)(*K), (C.c_double * 3)(*L), float(beta),
                                  float(CC), int(nbin), 1 if bound0 else 0, int(device)), "md_hspme_create")
        self.h = h
        self.natoms, self.K, self.L = int(natoms), K, L
        n = C.c_int()
        check(lib.md_hspme_num_coeffs(self.h, C.byref(n)), "md_hspme_num_coeffs")
        self.ncoef = n.value

    def __del__(self):
        if getattr(self, "h", None):
            lib.md_hspme_destroy(self.h)
            self.h = None

    @staticmethod
    def _ptr(t):
        return None if t is None else t.data_ptr()

    def energy(self, q, r, coeffs, forces=False, grads=False):
        """energy [C] (coeffs [C, ncoef] or [ncoef]) and, as asked, ik forces
        [C, N, 3] and the gradients dE/dq [C, N], dE/dr [C, N, 3], dE/dc [C, ncoef]."""
        torch = _torch()
        c = coeffs.detach().reshape(-1, self.ncoef).to(torch.float64).contiguous()
        q = q.detach().to(torch.float64).contiguous()
        r = r.detach().to(torch.float64).contiguous()
        nc, n, dev = c.shape[0], self.natoms, c.device
        e = torch.empty(nc, dtype=torch.float64, device=dev)
        F = torch.empty(nc, n, 3, dtype=torch.float64, device=dev) if forces else None
        gq = torch.empty(nc, n, dtype=torch.float64, device=dev) if grads else None
        gr = torch.empty(nc, n, 3, dtype=torch.float64, device=dev) if grads else None
        gc = torch.empty(nc, self.ncoef, dtype=torch.float64, device=dev) if grads else None
        P = self._ptr
        check(lib.md_hspme_energy(self.h, P(q), P(r), P(c), nc, P(e), P(F), P(gq), P(gr), P(gc),
                                  torch.cuda.current_stream(dev).cuda_stream), "md_hspme_energy")
        return {"energy": e, "forces": F, "dE_dq": gq, "dE_dr": gr, "dE_dc": gc}

    def force_error(self, q, r, coeffs, fref, grads=True):
        """L [C] = 1/N sum_i |F_i - fref_i|^2 of the ik forces against fref [N, 3] and,
        with grads, dL/dq [C, N], dL/dr [C, N, 3], dL/dc [C, ncoef]."""
        torch = _torch()
        c = coeffs.detach().reshape(-1, self.ncoef).to(torch.float64).contiguous()
        q = q.detach().to(torch.float64).contiguous()
        r = r.detach().to(torch.float64).contiguous()
        f = fref.detach().to(torch.float64).contiguous()
        nc, n, dev = c.shape[0], self.natoms, c.device
        loss = torch.empty(nc, dtype=torch.float64, device=dev)
        gq = torch.empty(nc, n, dtype=torch.float64, device=dev) if grads else None
        gr = torch.empty(nc, n, 3, dtype=torch.float64, device=dev) if grads else None
        gc = torch.empty(nc, self.ncoef, dtype=torch.float64, device=dev) if grads else None
        P = self._ptr
        check(lib.md_hspme_force_error(self.h, P(q), P(r), P(c), nc, P(f), P(loss), P(gq), P(gr), P(gc),
                                       torch.cuda.current_stream(dev).cuda_stream), "md_hspme_force_error")
        return {"loss": loss, "dL_dq": gq, "dL_dr": gr, "dL_dc": gc}


def hermite_spme_energy(q, r, coeffs, hspme):
    """Reciprocal energies [C] of the candidate bases coeffs [C, ncoef], as a
    torch.autograd.Function differentiable in q [N], r [N, 3] and coeffs (the
    gradients come from the hand-written adjoint in the same pass)."""
    torch = _torch()

    class _E(torch.autograd.Function):
        @staticmethod
        def forward(ctx, qq, rr, cc):
            out = hspme.energy(qq, rr, cc, grads=True)
            ctx.save_for_backward(out["dE_dq"], out["dE_dr"], out["dE_dc"])
            ctx.cshape = cc.shape
            return out["energy"]

        @staticmethod
        def backward(ctx, g):
            gq, gr, gc = ctx.saved_tensors
            g = g.reshape(-1)
            return ((g[:, None] * gq).sum(0), (g[:, None, None] * gr).sum(0),
                    (g[:, None] * gc).reshape(ctx.cshape))

    return _E.apply(q, r, coeffs)


def hermite_spme_force_error(q, r, coeffs, fref, hspme):
    """Force-error functional [C] (1/N sum |F_ik - fref|^2 per candidate) as a
    torch.autograd.Function differentiable in q, r and coeffs (second adjoint of
    the SPME chain, md_hspme_force_error); fref is a constant."""
    torch = _torch()

    class _L(torch.autograd.Function):
        @staticmethod
        def forward(ctx, qq, rr, cc):
            out = hspme.force_error(qq, rr, cc, fref, grads=True)
            ctx.save_for_backward(out["dL_dq"], out["dL_dr"], out["dL_dc"])
            ctx.cshape = cc.shape
            return out["loss"]

        @staticmethod
        def backward(ctx, g):
            gq, gr, gc = ctx.saved_tensors
            g = g.reshape(-1)
            return ((g[:, None] * gq).sum(0), (g[:, None, None] * gr).sum(0),
                    (g[:, None] * gc).reshape(ctx.cshape))

    return _L.apply(q, r, coeffs)


def bspline_initial_basis(CC, nbin, order, bound0=False):
    """The B-spline starting point of optiBasis/compute_basis.py:80-93: the
    centred cardinal B-spline of `order` and its slope at the knots j CC/nbin,
    divided by its value at 0 (knot 0 dropped; the last knot too when
    bound0)."""
    from math import comb, factorial
    n = int(order)

    def val_der(x):
        y = x + n / 2.0
        if not (-n / 2.0 < x < n / 2.0):
            return 0.0, 0.0
        v = sum((-1) ** j * comb(n, j) * max(y - j, 0.0) ** (n - 1) for j in range(n + 1)) / factorial(n - 1)
        d = sum((-1) ** j * comb(n, j) * max(y - j, 0.0) ** (n - 2) for j in range(n + 1)) / factorial(n - 2)
        return v, d

    h = CC / nbin
    vd = [val_der(j * h) for j in range(nbin + 1)]
    s = vd[0][0]
    v = np.array([a for a, _ in vd[1:]]) / s
    d = np.array([b for _, b in vd[1:]]) / s
    if bound0:
        v, d = v[:-1], d[:-1]
    return np.concatenate([v, d])
