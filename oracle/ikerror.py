"""ORACLE -- test infrastructure only.  numpy restatement of the optiBasis
ik-SPME force-error functional and its gradient with respect to the
interpolation-basis coefficients.

Reference: IkError.prepare_sum / prepare_sum_deriv / estimate / estimate_deriv
(optiBasis/IkError.py:32-136), HermiteLossFunc(_Bound0).value/deriv
(optiBasis/IkError.py:166-260), HermiteBasisHatComput_Norm1(_Bound0)
(optiBasis/HatComput.py:155-300), symm_hermite (optiBasis/Hermite.py:112-130),
unpack_v_d (optiBasis/basis_common.py:13-19).  Pinned against the values
and gradients of the reference's own Python in tests/golden/ikerror_cases.json.

The functional, for mesh K_d, box L_d, splitting beta, cut l_cut:
    sum_o1 = 1/(2 pi V)^2  sum_{m != 0, |m_d| <= K_d/2}  2 |G(m)|^2  sum_d T_d(m_d)
    T_d(m) = sum_{l != 0, |l| <= l_cut} phi_d(|m + l K_d|)^2 / phi_d(|m|)^2
    |G(m)|^2 = 16 pi^2 exp(-2 pi^2 |m*|^2 / beta^2) / |m*|^2,  m* = (m_d / L_d)
    error = conv * sqrt(sum_o1 q2^2 / N)
where phi_d is the real DFT of the over-sampled basis along axis d.  Since
T_d depends on m_d alone, sum_o1 = sum_d sum_m W_d(m) T_d(m) with
W_d(m) = sum over the other two indices of 2 |G|^2 (m != 0) -- the form the
GPU uses; this restatement keeps both forms (tests compare them).
"""
import numpy as np

CONVERSION = 138.93545756169981341199  # optiBasis/IkError.py:25


# ---------------------------------------------------------------- basis
def _h00(t): return (1 + 2 * t) * (1 - t) * (1 - t)
def _h01(t): return t * t * (3.0 - 2.0 * t)
def _h10(t): return t * (1 - t) * (1 - t)
def _h11(t): return t * t * (t - 1)


def hermite_pair(x, knot, h):
    """Cubic Hermite value- and slope-basis functions of knot `knot` (spacing
    h) at x: left piece on ((knot-1)h, knot h), right piece on [knot h,
    (knot+1)h); zero elsewhere (optiBasis/Hermite.py:30-110)."""
    s = x / h
    inside = (s > knot - 1) & (s < knot + 1)
    left = x < knot * h
    tl, tr = s - (knot - 1), s - knot
    v = np.where(left, _h01(tl), _h00(tr))
    d = np.where(left, _h11(tl) * h, _h10(tr) * h)
    return np.where(inside, v, 0.0), np.where(inside, d, 0.0)


def symmetric_pair(x, knot, h):
    """Even value basis V_j(x) + V_{-j}(x) and the slope basis D_j(x) -
    D_{-j}(x) (odd slopes keep the function even); knot 0 alone for j = 0."""
    v, d = hermite_pair(x, knot, h)
    if knot == 0:
        return v, d
    v2, d2 = hermite_pair(x, -knot, h)
    return v + v2, d - d2


def sample_grid(K, over_smpl):
    """The over-sampled periodic grid of optiBasis/HatComput.py:169-173:
    x_n = n K/M on [0, K), folded to x - K above K/2."""
    M = K * over_smpl
    x = np.arange(0, K, float(K) / float(M))
    return np.where(x > float(K / 2.0), x - K, x)


def basis_hats(CC, nbin, K, over_smpl, bound0, kmax):
    """hat0[k], hats[b][k] for k = 0..kmax: real part of the normalised DFT
    of each sampled basis function.  Order of b: value knots then slope
    knots, i.e. the coefficient vector [v_1..v_n, d_1..d_n] with n = nbin
    (knots 1..nbin, the last truncated to |x| <= CC) or nbin - 1 (bound0:
    knots 1..nbin-1, vanishing boundary).  Knot 0 has value 1 and slope 0
    (the Norm1 normalisation), so it is the constant part hat0."""
    h = CC / nbin
    x = sample_grid(K, over_smpl)
    M = len(x)

    def hat(f):
        return (np.fft.fft(f) / M).real[: kmax + 1]

    v0, _ = symmetric_pair(x, 0, h)
    hat0 = hat(v0)
    knots = list(range(1, nbin if bound0 else nbin + 1))
    hv, hd = [], []
    for j in knots:
        v, d = symmetric_pair(x, j, h)
        if j == nbin:
            keep = (x <= CC) & (x >= -CC)
            v, d = np.where(keep, v, 0.0), np.where(keep, d, 0.0)
        hv.append(hat(v))
        hd.append(hat(d))
    return hat0, np.array(hv + hd)


# ---------------------------------------------------------------- sums
def g2_grid(K, L, beta):
    """2 |G(m)|^2 on the (K0+1)(K1+1)(K2+1) grid |m_d| <= K_d/2 (0 at m = 0)."""
    ax = [np.arange(-(k // 2), k // 2 + 1) / l for k, l in zip(K, L)]
    m0, m1, m2 = np.meshgrid(*ax, indexing="ij")
    mm = m0 * m0 + m1 * m1 + m2 * m2
    with np.errstate(divide="ignore", invalid="ignore"):
        expp = np.exp(-np.pi * np.pi / (beta * beta) * mm) / mm
        g2 = 16 * np.pi * np.pi * mm * expp * expp
    g2[mm == 0] = 0.0
    return 2.0 * g2


def axis_weights(K, L, beta):
    """W_d(m) = sum over the other two indices of 2 |G|^2, m = -K_d/2..K_d/2."""
    g = g2_grid(K, L, beta)
    return [g.sum(axis=(1, 2)), g.sum(axis=(0, 2)), g.sum(axis=(0, 1))]


class IkErrorOracle:
    """HermiteLossFunc / HermiteLossFunc_Bound0 restated."""

    def __init__(self, CC, nbin, beta, K, L, q2, natoms, l_cut=10, bound0=False, over_smpl=None):
        self.K = [int(k) for k in K]
        self.L = np.asarray(L, dtype=float)
        self.beta, self.q2, self.natoms, self.l_cut = float(beta), float(q2), float(natoms), int(l_cut)
        self.V = float(np.prod(self.L))
        os_ = int(400 * (nbin / CC)) if over_smpl is None else int(over_smpl)
        self.hats = []
        for k in self.K:
            kmax = k // 2 + self.l_cut * k
            self.hats.append(basis_hats(CC, nbin, k, os_, bound0, kmax))
        self.W = axis_weights(self.K, self.L, self.beta)
        self.ncoef = self.hats[0][1].shape[0]

    def phi(self, d, vv):
        hat0, hb = self.hats[d]
        return hat0 + np.asarray(vv, dtype=float) @ hb

    def _terms(self, d, vv):
        k = self.K[d]
        m = np.arange(-(k // 2), k // 2 + 1)
        phi = self.phi(d, vv)
        hb = self.hats[d][1]
        ls = [l for l in range(-self.l_cut, self.l_cut + 1) if l != 0]
        p0 = phi[np.abs(m)]
        b0 = hb[:, np.abs(m)]
        T = np.zeros(len(m))
        dT = np.zeros((hb.shape[0], len(m)))
        for l in ls:
            idx = np.abs(m + l * k)
            pl, bl = phi[idx], hb[:, idx]
            T += pl * pl / (p0 * p0)
            dT += 2 * pl * bl / (p0 * p0) - 2 * pl * pl * b0 / (p0 * p0 * p0)
        return T, dT

    def sum_o1(self, vv):
        s = sum((self.W[d] * self._terms(d, vv)[0]).sum() for d in range(3))
        return s / (2 * np.pi * self.V * 2 * np.pi * self.V)

    def value(self, vv):
        return float(np.sqrt(self.sum_o1(vv) * self.q2 * self.q2 / self.natoms) * CONVERSION)

    def deriv(self, vv):
        s = self.sum_o1(vv)
        ds = sum(self.W[d] @ self._terms(d, vv)[1].T for d in range(3))
        ds = ds / (2 * np.pi * self.V * 2 * np.pi * self.V)
        return ds * 0.5 / np.sqrt(s) * np.sqrt(self.q2 * self.q2 / self.natoms) * CONVERSION

    def sum_o1_direct(self, vv):
        """The unfactorised triple sum, for small meshes."""
        g = g2_grid(self.K, self.L, self.beta)
        T = [self._terms(d, vv)[0] for d in range(3)]
        tot = g * (T[0][:, None, None] + T[1][None, :, None] + T[2][None, None, :])
        return tot.sum() / (2 * np.pi * self.V * 2 * np.pi * self.V)


def bspline_initial_basis(CC, nbin, order, bound0):
    """Cardinal B-spline of `order`, centred, sampled at the knots and
    normalised to 1 at 0 (optiBasis/compute_basis.py:80-93): v_j, d_j."""
    from math import comb, factorial

    def M(n, x):  # centred cardinal B-spline and its derivative (explicit sum)
        y = x + n / 2.0
        val = sum((-1) ** j * comb(n, j) * max(y - j, 0.0) ** (n - 1) for j in range(n + 1)) / factorial(n - 1)
        der = sum((-1) ** j * comb(n, j) * max(y - j, 0.0) ** (n - 2) for j in range(n + 1)) / factorial(n - 2)
        inside = -n / 2.0 < x < n / 2.0
        return (val, der) if inside else (0.0, 0.0)

    h = CC / nbin
    xs = [j * h for j in range(nbin + 1)]
    vals = [M(order, x) for x in xs]
    s = vals[0][0]
    v = np.array([a for a, _ in vals[1:]]) / s
    d = np.array([b for _, b in vals[1:]]) / s
    if bound0:
        v, d = v[:-1], d[:-1]
    return np.concatenate([v, d])
