"""ORACLE (test infrastructure only): SPME with optiBasis's Hermite
interpolation basis and its adjoints, restated in numpy for small systems,
as the checker of md.error_b200/csrc/hspme.cu.

The basis is optiBasis's symmetric piecewise cubic Hermite basis
(optiBasis/Hermite.py:6-130, optiBasis/HatComput.py:155-300): phi(x) = p(|x|)
on |x| < CC, value 1 and slope 0 at 0, coefficients [v_1..v_n, d_1..d_n] at
the knots j CC/nbin.  The SPME is ElectrostaticInteraction_rec_BSpline
(longRange.hetero/profile.test/template/tools/real.error/src/EleRecBSpline.cpp:
393-536, ik) with the B-spline replaced by phi and the interpolation factor of
calB (:729-796) formed from phi's integer samples.  Pure-Python loops over
atoms and stencil points: a few dozen atoms on small meshes.
"""
import numpy as np


class HermiteSPME:
    def __init__(self, K, L, beta, CC, nbin, bound0=False):
        self.K = tuple(int(k) for k in K)
        self.L = np.asarray(L, float)
        self.beta = float(beta)
        self.CC = float(CC)
        self.nbin = int(nbin)
        self.nk = self.nbin - 1 if bound0 else self.nbin
        self.ncoef = 2 * self.nk
        self.h = self.CC / self.nbin
        self.half = int(np.ceil(self.CC - 1e-12))
        self.S = 2 * self.half
        mi = [np.fft.fftfreq(k, 1.0 / k) for k in self.K]
        self.mv = np.meshgrid(*[mi[d] / self.L[d] for d in range(3)], indexing="ij")
        m2 = self.mv[0] ** 2 + self.mv[1] ** 2 + self.mv[2] ** 2
        self.zero = m2 == 0
        m2[self.zero] = 1.0
        self.m2 = m2

    # phi, phi' and dphi/dc at x
    def phi(self, c, x):
        nk, h = self.nk, self.h
        dc = np.zeros(self.ncoef)
        ax = abs(x)
        if not ax < self.CC:
            return 0.0, 0.0, dc
        V = [1.0] + list(c[:nk]) + [0.0]
        D = [0.0] + list(c[nk:]) + [0.0]
        j = min(int(ax / h), self.nbin - 1)
        t = ax / h - j
        hv = [(1 + 2 * t) * (1 - t) ** 2, t * (1 - t) ** 2, t * t * (3 - 2 * t), t * t * (t - 1)]
        hd = [6 * t * (t - 1), (3 * t - 1) * (t - 1), 6 * t * (1 - t), t * (3 * t - 2)]
        V0, D0 = V[j], D[j]
        V1 = V[j + 1] if j + 1 <= nk else 0.0
        D1 = D[j + 1] if j + 1 <= nk else 0.0
        p = hv[0] * V0 + hv[1] * h * D0 + hv[2] * V1 + hv[3] * h * D1
        dp = (hd[0] * V0 + hd[1] * h * D0 + hd[2] * V1 + hd[3] * h * D1) / h
        if 1 <= j <= nk:
            dc[j - 1] += hv[0]
            dc[nk + j - 1] += hv[1] * h
        if j + 1 <= nk:
            dc[j] += hv[2]
            dc[nk + j] += hv[3] * h
        return p, (dp if x >= 0 else -dp), dc

    def _stencil(self, c, r):
        out = []
        for d in range(3):
            f = r[d] / self.L[d]
            f -= np.floor(f)
            u = self.K[d] * f
            k0 = int(np.floor(u)) - self.half + 1
            out.append([(k0 + j,) + self.phi(c, u - (k0 + j)) for j in range(self.S)])
        return out

    def _influence(self, c):
        bf, dbf = [], []
        for d in range(3):
            m = np.arange(self.K[d])
            b = np.zeros(self.K[d])
            db = np.zeros((self.ncoef, self.K[d]))
            for k in range(-self.half, self.half + 1):
                v, _, dc = self.phi(c, float(k))
                cs = np.cos(2 * np.pi * m * k / self.K[d])
                b += v * cs
                db += dc[:, None] * cs[None, :]
            bf.append(b)
            dbf.append(db)
        V = float(np.prod(self.L))
        G = np.exp(-np.pi ** 2 * self.m2 / self.beta ** 2) / (np.pi * V * self.m2)
        G = G / (bf[0][:, None, None] ** 2 * bf[1][None, :, None] ** 2 * bf[2][None, None, :] ** 2)
        G[self.zero] = 0.0
        return G, bf, dbf

    def _spread(self, c, r, amp):
        Q = np.zeros((amp.shape[1],) + self.K)
        for i in range(r.shape[0]):
            st = self._stencil(c, r[i])
            for a in st[0]:
                for b in st[1]:
                    for e in st[2]:
                        Q[:, a[0] % self.K[0], b[0] % self.K[1], e[0] % self.K[2]] += amp[i] * a[1] * b[1] * e[1]
        return Q

    def _nyq(self, d):
        m = np.ones(self.K)
        idx = [slice(None)] * 3
        idx[d] = self.K[d] // 2
        if self.K[d] % 2 == 0:
            m[tuple(idx)] = 0.0
        return m

    def _contract(self, c, q, r, field):
        """sum_i q_i sum_k W_i s_i(k) with s_i(k) = field(i, k): its derivatives
        in q_i (without the q_i), r_i and c."""
        n = r.shape[0]
        dq, dr, dc = np.zeros(n), np.zeros((n, 3)), np.zeros(self.ncoef)
        kl = self.K / self.L
        for i in range(n):
            st = self._stencil(c, r[i])
            for a in st[0]:
                for b in st[1]:
                    for e in st[2]:
                        p = (a[0] % self.K[0], b[0] % self.K[1], e[0] % self.K[2])
                        s = field(i, p)
                        dq[i] += a[1] * b[1] * e[1] * s
                        dr[i] += q[i] * s * np.array([a[2] * kl[0] * b[1] * e[1], b[2] * kl[1] * a[1] * e[1],
                                                      e[2] * kl[2] * a[1] * b[1]])
                        dc += q[i] * s * (a[3] * b[1] * e[1] + b[3] * a[1] * e[1] + e[3] * a[1] * b[1])
        return dq, dr, dc

    def forward(self, c, q, r):
        """(E, F [N,3], state) of candidate c."""
        G, bf, dbf = self._influence(c)
        Q = self._spread(c, r, q[:, None])[0]
        Qh = np.fft.fftn(Q)
        E = 0.5 * float((G * np.abs(Qh) ** 2).sum())
        Kt = Q.size
        fld = [np.fft.ifftn(1j * 2 * np.pi * self.mv[d] * G * self._nyq(d) * Qh).real * Kt for d in range(3)]
        pot = np.fft.ifftn(G * Qh).real * Kt
        F = np.zeros((r.shape[0], 3))
        for i in range(r.shape[0]):
            st = self._stencil(c, r[i])
            for a in st[0]:
                for b in st[1]:
                    for e in st[2]:
                        w = a[1] * b[1] * e[1]
                        p = (a[0] % self.K[0], b[0] % self.K[1], e[0] % self.K[2])
                        for d in range(3):
                            F[i, d] -= q[i] * w * fld[d][p]
        return E, F, dict(G=G, bf=bf, dbf=dbf, Qh=Qh, fld=fld, pot=pot)

    def energy_grad(self, c, q, r):
        """E, F, dE/dq, dE/dr, dE/dc (hspme.cu's adjoint, restated)."""
        E, F, st = self.forward(c, q, r)
        dq, dr, dcW = self._contract(c, q, r, lambda i, p: st["pot"][p])
        P = [(st["G"] * np.abs(st["Qh"]) ** 2).sum(axis=tuple(x for x in range(3) if x != d)) for d in range(3)]
        dcG = -sum((st["dbf"][d] * (P[d] / st["bf"][d])[None, :]).sum(1) for d in range(3))
        return E, F, dq, dr, dcW + dcG

    def force_error_grad(self, c, q, r, fref):
        """L = 1/N sum |F - fref|^2 and dL/dq, dL/dr, dL/dc."""
        E, F, st = self.forward(c, q, r)
        n = r.shape[0]
        L = float(((F - fref) ** 2).sum() / n)
        R = 2 * (F - fref) / n
        B = self._spread(c, r, -q[:, None] * R)
        Bh = np.fft.fftn(B, axes=(1, 2, 3))
        G, Qh = st["G"], st["Qh"]
        lam = np.fft.ifftn(-sum(1j * 2 * np.pi * self.mv[d] * G * self._nyq(d) * Bh[d] for d in range(3))).real
        lam *= Q_size(self.K)
        H = np.real(sum(np.conj(Bh[d]) * 1j * 2 * np.pi * self.mv[d] * self._nyq(d) * Qh for d in range(3))) * G
        PH = [H.sum(axis=tuple(x for x in range(3) if x != d)) for d in range(3)]
        dcG = -2 * sum((st["dbf"][d] * (PH[d] / st["bf"][d])[None, :]).sum(1) for d in range(3))
        dq1, dr1, dc1 = self._contract(c, q, r, lambda i, p: lam[p])
        fld = st["fld"]
        dq2, dr2, dc2 = self._contract(c, q, r, lambda i, p: -(R[i, 0] * fld[0][p] + R[i, 1] * fld[1][p]
                                                                 + R[i, 2] * fld[2][p]))
        return L, dq1 + dq2, dr1 + dr2, dc1 + dc2 + dcG


def Q_size(K):
    return int(np.prod(K))
