"""ORACLE -- test infrastructure only (ctypes wrapper of oracle/liboracle.so).

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg, as the checker; the product package never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


if not os.path.exists(LIB):
    build()
_lib = C.CDLL(LIB)

P = C.POINTER
f32, f64, i32, i64, u32, u64 = C.c_float, C.c_double, C.c_int, C.c_int64, C.c_uint32, C.c_uint64


class LvParams(C.Structure):
    _fields_ = [("dt", f64), ("temperature", f64), ("gamma_t", f64), ("tau_p", f64),
                ("kappa_t", f64), ("p_ref", f64 * 3), ("npt_dirs", i32), ("seed", u64),
                ("skin", f64), ("eps", f64), ("sigma", f64), ("shift", f64)]


_sigs = {
    "orc_box_inverse_f32": (None, [P(f32), P(f32)]),
    "orc_decide_ncell": (i32, [P(f64), f64, i32, i32, P(i32)]),
    "orc_bin_f32": (None, [i32, P(f32), P(i32), P(f32), P(i32), P(u32)]),
    "orc_bin_f64": (None, [i32, P(f64), P(i32), P(f64), P(i32), P(u32)]),
    "orc_nlist_allpair_f32": (None, [i32, P(f32), P(f32), f32, P(f32), i32, P(i32), P(i32)]),
    "orc_nlist_allpair_f64": (None, [i32, P(f64), P(f64), f64, P(f64), i32, P(i32), P(i32)]),
    "orc_nlist_cellshift_f32": (None, [i32, P(f32), P(u32), f32, P(f32), P(i32), i32, P(i32), P(i32)]),
    "orc_lj_allpair_f64": (None, [i32, P(f64), P(f64), f64, f64, f64, P(f64), P(f32), P(f32), P(f64), P(f64)]),
    "orc_lattice_rcut_f32": (f32, [f32, f32, f32, P(f32), P(f32), i32, i32, i32]),
    "orc_assign_rcut_f32": (None, [i32, P(f32), P(f32), P(f32), i32, i32, i32, P(f32)]),
    "orc_normals4": (None, [u64, u64, u32, P(f64)]),
    "orc_md_langevin_run": (i32, [i32, P(f64), P(f64), P(f64), P(f32), P(f32), i32, i32, i32, P(f64),
                                  P(LvParams), P(f64), i32, i32, P(f64), P(i64)]),
    "orc_md_nhc_run": (i32, [i32, P(f64), P(f64), P(f64), P(f32), P(f64), P(LvParams), i32, i32, i32, P(f64),
                             P(f64), P(i64)]),
    "orc_md_nhc_npt_run": (i32, [i32, P(f64), P(f64), P(f64), P(f32), P(f64), P(LvParams), f64, i32, i32,
                                 P(f64), P(f64)]),
    "orc_num_threads": (i32, []),
    "orc_philox4x32_10": (None, [P(u32), P(u32), P(u32)]),
}
for _n, (_r, _a) in _sigs.items():
    _f = getattr(_lib, _n)
    _f.restype = _r
    _f.argtypes = _a


def _p(a, t):
    return a.ctypes.data_as(P(t))


def box_inverse_f32(box):
    b = np.ascontiguousarray(box, np.float32)
    out = np.empty(3, np.float32)
    _lib.orc_box_inverse_f32(_p(b, f32), _p(out, f32))
    return out


def decide_ncell(box, cell_size, bdir=7, divide=1):
    b = np.ascontiguousarray(box, np.float64)
    nc = np.empty(3, np.int32)
    mode = _lib.orc_decide_ncell(_p(b, f64), float(cell_size), bdir, divide, _p(nc, i32))
    return tuple(int(x) for x in nc), bool(mode)


def bin_f32(pos, box, ncell):
    """normalise + cell index (binary32); returns (pos_wrapped, image, cell)."""
    p = np.ascontiguousarray(pos, np.float32).copy()
    n = p.shape[0]
    img = np.zeros((n, 3), np.int32)
    b = np.ascontiguousarray(box, np.float32)
    nc = np.ascontiguousarray(ncell, np.int32)
    cell = np.empty(n, np.uint32)
    _lib.orc_bin_f32(n, _p(p, f32), _p(img, i32), _p(b, f32), _p(nc, i32), _p(cell, u32))
    return p, img, cell


def bin_f64(pos, box, ncell):
    p = np.ascontiguousarray(pos, np.float64).copy()
    n = p.shape[0]
    img = np.zeros((n, 3), np.int32)
    b = np.ascontiguousarray(box, np.float64)
    nc = np.ascontiguousarray(ncell, np.int32)
    cell = np.empty(n, np.uint32)
    _lib.orc_bin_f64(n, _p(p, f64), _p(img, i32), _p(b, f64), _p(nc, i32), _p(cell, u32))
    return p, img, cell


def _csr(counts, pairs, cap):
    n = counts.shape[0]
    if (counts > cap).any():
        raise RuntimeError("oracle list capacity exceeded")
    rows = [pairs[i * cap:i * cap + counts[i]] for i in range(n)]
    return counts.copy(), (np.concatenate(rows) if n else np.empty(0, np.int32))


def nlist_allpair_f32(pos, rcut, skin, box, cap=1024):
    p = np.ascontiguousarray(pos, np.float32)
    n = p.shape[0]
    rc = np.ascontiguousarray(rcut, np.float32)
    b = np.ascontiguousarray(box, np.float32)
    counts = np.empty(n, np.int32)
    pairs = np.empty(n * cap, np.int32)
    _lib.orc_nlist_allpair_f32(n, _p(p, f32), _p(rc, f32), float(np.float32(skin)), _p(b, f32), cap,
                               _p(counts, i32), _p(pairs, i32))
    return _csr(counts, pairs, cap)


def nlist_allpair_f64(pos, rcut, skin, box, cap=1024):
    p = np.ascontiguousarray(pos, np.float64)
    n = p.shape[0]
    rc = np.ascontiguousarray(rcut, np.float64)
    b = np.ascontiguousarray(box, np.float64)
    counts = np.empty(n, np.int32)
    pairs = np.empty(n * cap, np.int32)
    _lib.orc_nlist_allpair_f64(n, _p(p, f64), _p(rc, f64), float(skin), _p(b, f64), cap,
                               _p(counts, i32), _p(pairs, i32))
    return _csr(counts, pairs, cap)


def nlist_cellshift_f32(pos, cell, rlist, box, ncell, cap=1024):
    p = np.ascontiguousarray(pos, np.float32)
    n = p.shape[0]
    c = np.ascontiguousarray(cell, np.uint32)
    b = np.ascontiguousarray(box, np.float32)
    nc = np.ascontiguousarray(ncell, np.int32)
    counts = np.empty(n, np.int32)
    pairs = np.empty(n * cap, np.int32)
    _lib.orc_nlist_cellshift_f32(n, _p(p, f32), _p(c, u32), float(np.float32(rlist)), _p(b, f32),
                                 _p(nc, i32), cap, _p(counts, i32), _p(pairs, i32))
    return _csr(counts, pairs, cap)


def lj_allpair_f64(pos, rcut, box, eps=1.0, sigma=1.0, shift=0.0, pos32=None, box32=None):
    """FP64 all-pairs LJ; returns (force[N,3], stats[E, Wxx, Wyy, Wzz])."""
    p = np.ascontiguousarray(pos, np.float64)
    n = p.shape[0]
    rc = np.ascontiguousarray(rcut, np.float64)
    b = np.ascontiguousarray(box, np.float64)
    F = np.empty((n, 3), np.float64)
    st = np.empty(4, np.float64)
    p32 = None if pos32 is None else np.ascontiguousarray(pos32, np.float32)
    b32 = None if box32 is None else np.ascontiguousarray(box32, np.float32)
    _lib.orc_lj_allpair_f64(n, _p(p, f64), _p(rc, f64), eps, sigma, shift, _p(b, f64),
                            None if p32 is None else _p(p32, f32), None if b32 is None else _p(b32, f32),
                            _p(F, f64), _p(st, f64))
    return F, st


def lj_allpair_typed(pos, rcut, box, types, pairs, pos32=None, box32=None):
    """All-pairs non-bonded forces with atom types; pairs = {(t0, t1): params} (symmetric)
    with params (eps, sigma, shift) for LJ 6-12 or (kind, (p0, p1, p2, p3)) for the other
    kinds (1 LJ 6-12, 5 LJ 6-12 B, 3 CosTail); other pairs take no force.
    Returns (force[N,3], stats[E, Wxx, Wyy, Wzz])."""
    p = np.ascontiguousarray(pos, np.float64)
    n = p.shape[0]
    t = np.ascontiguousarray(types, np.int32)
    nt = int(max(max(max(k) for k in pairs) + 1, t.max() + 1))
    tab = np.zeros((nt, nt, 6)); on = np.zeros((nt, nt), np.int32)
    for (a, b), v in pairs.items():
        kind, q = (1, tuple(v)) if not isinstance(v[0], int) or len(v) != 2 else v
        q = np.pad(np.asarray(q, float), (0, 6 - len(q)))
        tab[a, b] = tab[b, a] = q
        on[a, b] = on[b, a] = kind
    rc = np.ascontiguousarray(rcut, np.float64)
    b = np.ascontiguousarray(box, np.float64)
    F = np.empty((n, 3)); st = np.empty(4)
    p32 = None if pos32 is None else np.ascontiguousarray(pos32, np.float32)
    b32 = None if box32 is None else np.ascontiguousarray(box32, np.float32)
    _lib.orc_lj_allpair_typed(n, _p(p, f64), _p(rc, f64), _p(t, i32), nt, _p(tab, f64), _p(on, i32), _p(b, f64),
                              None if p32 is None else _p(p32, f32), None if b32 is None else _p(b32, f32),
                              _p(F, f64), _p(st, f64))
    return F, st


def assign_rcut_f32(pos, box, lattice):
    p = np.ascontiguousarray(pos, np.float32)
    b = np.ascontiguousarray(box, np.float32)
    lat = np.ascontiguousarray(lattice, np.float32)
    nx, ny, nz = lat.shape
    out = np.empty(p.shape[0], np.float32)
    _lib.orc_assign_rcut_f32(p.shape[0], _p(p, f32), _p(b, f32), _p(lat, f32), nx, ny, nz, _p(out, f32))
    return out


def normals4(seed, step, idx):
    out = np.empty(4, np.float64)
    _lib.orc_normals4(seed, step, idx, _p(out, f64))
    return out


def md_langevin_run(pos, vel, box, nsteps, *, dt, temperature, gamma_t, skin, rcut=None,
                    lattice=None, tau_p=0.0, kappa_t=0.0, p_ref=(0, 0, 0), npt_dirs=0, seed=1,
                    eps=1.0, sigma=1.0, shift=0.0, pcorr=None, cap=1024, mass=None):
    """CPU FP64 Langevin MD; returns dict(pos, vel, box, stats, rebuilds, max_list, status)."""
    p = np.ascontiguousarray(pos, np.float64).copy()
    v = np.ascontiguousarray(vel, np.float64).copy()
    n = p.shape[0]
    b = np.ascontiguousarray(box, np.float64).copy()
    prm = LvParams()
    prm.dt, prm.temperature, prm.gamma_t, prm.tau_p, prm.kappa_t = dt, temperature, gamma_t, tau_p, kappa_t
    for d in range(3):
        prm.p_ref[d] = p_ref[d]
    prm.npt_dirs, prm.seed, prm.skin, prm.eps, prm.sigma, prm.shift = npt_dirs, seed, skin, eps, sigma, shift
    rc = None if rcut is None else np.ascontiguousarray(rcut, np.float32)
    lat = None if lattice is None else np.ascontiguousarray(lattice, np.float32)
    nx, ny, nz = (lat.shape if lat is not None else (0, 0, 0))
    m = None if mass is None else np.ascontiguousarray(mass, np.float64)
    pc = None if pcorr is None else np.ascontiguousarray(pcorr, np.float64)
    stats = np.zeros(7, np.float64)
    cnt = np.zeros(2, np.int64)
    status = _lib.orc_md_langevin_run(n, _p(p, f64), _p(v, f64), None if m is None else _p(m, f64),
                                      None if rc is None else _p(rc, f32), None if lat is None else _p(lat, f32),
                                      nx, ny, nz, _p(b, f64), C.byref(prm), None if pc is None else _p(pc, f64),
                                      int(nsteps), int(cap), _p(stats, f64), _p(cnt, i64))
    return dict(pos=p, vel=v, box=b, stats=stats, rebuilds=int(cnt[0]), max_list=int(cnt[1]), status=status)


def md_nhc_run(pos, vel, box, nsteps, *, dt, temperature, tau_t, skin, rcut, remove_com=True,
               eps=1.0, sigma=1.0, shift=0.0, cap=1024, mass=None):
    """CPU FP64 Nose-Hoover-chain velocity-Verlet MD (the lj.nhc-xtc step);
    returns dict(pos, vel, stats, nhc, rebuilds, max_list, status)."""
    p = np.ascontiguousarray(pos, np.float64).copy()
    v = np.ascontiguousarray(vel, np.float64).copy()
    n = p.shape[0]
    b = np.ascontiguousarray(box, np.float64).copy()
    prm = LvParams()
    prm.dt, prm.temperature, prm.tau_p = dt, temperature, tau_t
    prm.skin, prm.eps, prm.sigma, prm.shift = skin, eps, sigma, shift
    rc = np.ascontiguousarray(rcut, np.float32)
    m = None if mass is None else np.ascontiguousarray(mass, np.float64)
    stats = np.zeros(7, np.float64)
    nhc = np.zeros(5, np.float64)
    cnt = np.zeros(2, np.int64)
    status = _lib.orc_md_nhc_run(n, _p(p, f64), _p(v, f64), None if m is None else _p(m, f64), _p(rc, f32),
                                 _p(b, f64), C.byref(prm), 1 if remove_com else 0, int(nsteps), int(cap),
                                 _p(stats, f64), _p(nhc, f64), _p(cnt, i64))
    return dict(pos=p, vel=v, stats=stats, nhc=nhc, rebuilds=int(cnt[0]), max_list=int(cnt[1]), status=status)


def md_nhc_npt_run(pos, vel, box, nsteps, *, dt, temperature, tau_t, p_ref, tau_p, skin, rcut, pcorr=0.0,
                   eps=1.0, sigma=1.0, shift=0.0, cap=1024, mass=None):
    """CPU FP64 isobaric Nose-Hoover chain (MTK step of the reference operators);
    returns dict(pos, vel, box, stats, state, status)."""
    p = np.ascontiguousarray(pos, np.float64).copy()
    v = np.ascontiguousarray(vel, np.float64).copy()
    n = p.shape[0]
    b = np.ascontiguousarray(box, np.float64).copy()
    prm = LvParams()
    prm.dt, prm.temperature, prm.gamma_t, prm.tau_p = dt, temperature, tau_t, tau_p
    prm.p_ref[0] = p_ref
    prm.skin, prm.eps, prm.sigma, prm.shift = skin, eps, sigma, shift
    rc = np.ascontiguousarray(rcut, np.float32)
    m = None if mass is None else np.ascontiguousarray(mass, np.float64)
    stats = np.zeros(7, np.float64)
    state = np.zeros(5, np.float64)
    status = _lib.orc_md_nhc_npt_run(n, _p(p, f64), _p(v, f64), None if m is None else _p(m, f64), _p(rc, f32),
                                     _p(b, f64), C.byref(prm), float(pcorr), int(nsteps), int(cap), _p(stats, f64),
                                     _p(state, f64))
    return dict(pos=p, vel=v, box=b, stats=stats, state=state, status=status)


def num_threads():
    return _lib.orc_num_threads()


def philox4x32_10(ctr, key):
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    out = np.empty(4, np.uint32)
    _lib.orc_philox4x32_10(_p(c, u32), _p(k, u32), _p(out, u32))
    return out


# ---------------------------------------------------------------- AdaptRCut
_lib2 = _lib
_sigs2 = {
    "orc_dp_bins": (None, [P(f64), f64, P(i32)]),
    "orc_dp_deposit": (None, [i32, P(f32), P(f64), P(i32), P(f64)]),
    "orc_dp_calculate": (None, [P(f64), P(i32), i32, P(f64)]),
    "orc_dft3d": (None, [P(i32), P(f64), i32]),
    "orc_gauss4": (f64, [i32, f64, f64, f64, f64]),
    "orc_arc_kernels": (None, [P(f64), P(i32), P(f64), i32, f64, f64, P(f64), P(f64), P(f64), P(f64)]),
    "orc_arc_error": (None, [P(f64), P(i32), i32, P(f64), P(f64), P(f64), P(f64), P(f64), P(f64)]),
    "orc_arc_calrcut": (None, [i32, P(f64), C.c_long, P(f64), f64, P(f64), P(i32), P(f64)]),
    "orc_arc_refine": (None, [P(i32), P(f64), C.c_long, P(f64), P(i32), P(f64), P(f64)]),
    "orc_pc_kernels": (None, [P(f64), P(i32), P(f64), i32, P(f64), P(f64), P(f64)]),
    "orc_pc_correction": (None, [P(f64), P(i32), i32, P(f64), P(f64), P(f64), P(f64), P(i32), P(f64)]),
}
for _n, (_r, _a) in _sigs2.items():
    _f = getattr(_lib2, _n)
    _f.restype = _r
    _f.argtypes = _a


def dp_bins(box, refh):
    b = np.ascontiguousarray(box, np.float64)
    n = np.empty(3, np.int32)
    _lib.orc_dp_bins(_p(b, f64), float(refh), _p(n, i32))
    return tuple(int(x) for x in n)


def dp_deposit(coord, box, n, profile=None):
    c = np.ascontiguousarray(coord, np.float32)
    b = np.ascontiguousarray(box, np.float64)
    nn = np.ascontiguousarray(n, np.int32)
    prof = np.zeros(tuple(n), np.float64) if profile is None else profile
    _lib.orc_dp_deposit(c.shape[0], _p(c, f32), _p(b, f64), _p(nn, i32), _p(prof, f64))
    return prof


def spme_ana_errmap(K, box, beta, order, rho1, rho2, charge=1.0, with_fconv=False):
    """ErrorEstimate_SPME_Ana::reinit + calError restated (oracle_errmap.c): error1,
    error2 as (K0, K1, K2, 2) arrays, the uncharged self error, and with with_fconv
    FConvRho1 as (4, 3, K0, K1, K2, 2) for k = -2, -1, 1, 2 (else None)."""
    KK = np.ascontiguousarray(K, np.int32)
    b = np.ascontiguousarray(box, np.float64)
    r1 = np.ascontiguousarray(rho1, np.float64).reshape(-1)
    r2 = np.ascontiguousarray(rho2, np.float64).reshape(-1)
    e1 = np.zeros(tuple(K) + (2,)); e2 = np.zeros(tuple(K) + (2,))
    self_ = C.c_double()
    fc = np.zeros((4, 3) + tuple(K) + (2,)) if with_fconv else None
    _lib.orc_spme_ana_errmap(_p(KK, i32), _p(b, f64), float(beta), int(order), _p(r1, f64), _p(r2, f64),
                             float(charge), _p(e1, f64), _p(e2, f64), C.byref(self_),
                             _p(fc, f64) if with_fconv else None)
    return e1, e2, self_.value, fc


def ref_spme_ana_errmap(K, box, beta, order, rho1, rho2, charge=1.0, with_fconv=False):
    """The reference's own ErrorEstimate_SPME_Ana (oracle/_ref/libref_errana.so), same
    returns as spme_ana_errmap."""
    lib = C.CDLL(os.path.join(REF_DIR, "libref_errana.so"))
    lib.ref_spme_ana_errmap.argtypes = [P(i32), P(f64), f64, i32, P(f64), P(f64), f64, P(f64), P(f64),
                                        P(f64), P(f64)]
    KK = np.ascontiguousarray(K, np.int32)
    b = np.ascontiguousarray(box, np.float64)
    r1 = np.ascontiguousarray(rho1, np.float64).reshape(-1)
    r2 = np.ascontiguousarray(rho2, np.float64).reshape(-1)
    e1 = np.zeros(tuple(K) + (2,)); e2 = np.zeros(tuple(K) + (2,))
    self_ = np.zeros(1)
    fc = np.zeros((4, 3) + tuple(K) + (2,)) if with_fconv else None
    lib.ref_spme_ana_errmap(_p(KK, i32), _p(b, f64), float(beta), int(order), _p(r1, f64), _p(r2, f64),
                            float(charge), _p(e1, f64), _p(e2, f64), _p(self_, f64),
                            _p(fc, f64) if with_fconv else None)
    return e1, e2, float(self_[0]), fc


def dft3d(data, sign):
    """in-place unnormalised 3D DFT of a complex128 array"""
    d = np.ascontiguousarray(data, np.complex128).copy()
    n = np.array(d.shape, np.int32)
    _lib.orc_dft3d(_p(n, i32), d.ctypes.data_as(P(f64)), int(sign))
    return d


def gauss4(kind, k, xlo, xup, tol):
    return _lib.orc_gauss4(kind, k, xlo, xup, tol)


def arc_kernels(box, n, rc, eps=1.0, sigma=1.0):
    b = np.ascontiguousarray(box, np.float64)
    nn = np.ascontiguousarray(n, np.int32)
    rcl = np.ascontiguousarray(rc, np.float64)
    nrc = len(rcl)
    shp = (nrc,) + tuple(n)
    s1, sx, sy, sz = (np.zeros(shp) for _ in range(4))
    _lib.orc_arc_kernels(_p(b, f64), _p(nn, i32), _p(rcl, f64), nrc, eps, sigma, _p(s1, f64), _p(sx, f64),
                         _p(sy, f64), _p(sz, f64))
    return s1, np.stack([sx, sy, sz])


def pc_kernels(box, n, rc):
    b = np.ascontiguousarray(box, np.float64)
    nn = np.ascontiguousarray(n, np.int32)
    rcl = np.ascontiguousarray(rc, np.float64)
    nrc = len(rcl)
    shp = (nrc,) + tuple(n)
    kx, ky, kz = (np.zeros(shp) for _ in range(3))
    _lib.orc_pc_kernels(_p(b, f64), _p(nn, i32), _p(rcl, f64), nrc, _p(kx, f64), _p(ky, f64), _p(kz, f64))
    return np.stack([kx, ky, kz])


def adapt_rcut(box, n, rc, rho, prec, nrefine=0, with_pc=True):
    """AdaptRCut::calError + calRCut + refineRCut (+ PressureCorrection) on profile rho."""
    b = np.ascontiguousarray(box, np.float64)
    nn = np.ascontiguousarray(n, np.int32)
    rcl = np.ascontiguousarray(rc, np.float64)
    nrc = len(rcl)
    s1, s2 = arc_kernels(box, n, rc)
    s1 = np.ascontiguousarray(s1)
    sx, sy, sz = (np.ascontiguousarray(s2[d]) for d in range(3))
    r = np.ascontiguousarray(rho, np.float64).reshape(n)
    err = np.zeros((nrc,) + tuple(n))
    _lib.orc_arc_error(_p(b, f64), _p(nn, i32), nrc, _p(s1, f64), _p(sx, f64), _p(sy, f64), _p(sz, f64),
                       _p(r, f64), _p(err, f64))
    nele = int(np.prod(n))
    rcut = np.zeros(tuple(n)); idx = np.zeros(tuple(n), np.int32); rerr = np.zeros(tuple(n))
    _lib.orc_arc_calrcut(nrc, _p(rcl, f64), nele, _p(err, f64), float(prec), _p(rcut, f64), _p(idx, i32),
                         _p(rerr, f64))
    for _ in range(nrefine):
        _lib.orc_arc_refine(_p(nn, i32), _p(rcl, f64), nele, _p(err, f64), _p(idx, i32), _p(rcut, f64),
                            _p(rerr, f64))
    out = dict(error=err, rcut=rcut, index=idx, result_error=rerr, s1k=s1, s2k=s2)
    if with_pc:
        K = pc_kernels(box, n, rc)
        kx, ky, kz = (np.ascontiguousarray(K[d]) for d in range(3))
        p = np.zeros(3)
        _lib.orc_pc_correction(_p(b, f64), _p(nn, i32), nrc, _p(kx, f64), _p(ky, f64), _p(kz, f64), _p(r, f64),
                               _p(idx, i32), _p(p, f64))
        out["pcorr"] = p
        out["pck"] = K
    return out


def fcorr_field(box, n, rc, rho):
    """ForceCorr::makeS2k + calError (FCR/src/ForceCorr.cu:150-262): the s2k kernel
    is AdaptRCut's for the single cutoff rc; field_d = IFFT(s2k_d FFT(rho) V/nele)/V.
    Returns the complex field (3, nx, ny, nz)."""
    n = tuple(int(v) for v in n)
    V = float(np.prod(box))
    nele = int(np.prod(n))
    _, s2 = arc_kernels(box, n, [rc])
    rk = dft3d(np.asarray(rho, np.float64).reshape(n).astype(np.complex128), -1) * (V / nele)
    out = np.empty((3,) + n, np.complex128)
    for d in range(3):
        out[d] = dft3d(rk * (1j * s2[d, 0]), +1) / V
    return out


def fcorr_assign(pos, box, n, field_re, prec_f32=True):
    """AssignForceCorr::assign (FCR/src/AssignForceCorr.cu:131-163): wrap the
    binary32 coordinate once, bin ix = int((x nx) / Lx) in binary32, take the
    bin's value (rounded to binary32 for the mixed path)."""
    p = np.asarray(pos, np.float32)
    L = np.asarray(box, np.float32)
    nn = np.asarray(n, np.int64)
    idx = []
    for d in range(3):
        x = p[:, d].copy()
        x = np.where(x < 0, (x + L[d]).astype(np.float32), np.where(x >= L[d], (x - L[d]).astype(np.float32), x))
        q = ((x * np.float32(nn[d])).astype(np.float32) / L[d]).astype(np.float32)
        i = np.clip(np.trunc(q).astype(np.int64), 0, nn[d] - 1)
        idx.append(i)
    b = idx[2] + nn[2] * (idx[1] + nn[1] * idx[0])
    v = np.stack([field_re[d].reshape(-1)[b] for d in range(3)], 1)
    return v.astype(np.float32).astype(np.float64) if prec_f32 else v


# ---------------------------------------------------------------- reference (compiled from its sources)
REF_DIR = os.path.join(HERE, "_ref")


def ref_available(name):
    return os.path.exists(os.path.join(REF_DIR, name))


def ref_adapt_rcut(box, n, rcmin, rcmax, rcstep, rho, prec, nrefine=0):
    """The reference's own AdaptRCut + PressureCorrection (oracle/_ref/libref_arc.so)."""
    lib = C.CDLL(os.path.join(REF_DIR, "libref_arc.so"))
    lib.ref_arc_run.argtypes = [P(f64), P(i32), f64, f64, f64, P(f64), f64, i32, P(f64), P(f64), P(i32),
                                P(f64), P(f64)]
    b = np.ascontiguousarray(box, np.float64)
    nn = np.ascontiguousarray(n, np.int32)
    r = np.ascontiguousarray(rho, np.float64).reshape(n)
    nrc = len(np.arange(rcmin, rcmax + 1e-12, rcstep))
    err = np.zeros((nrc,) + tuple(n)); rcut = np.zeros(tuple(n)); idx = np.zeros(tuple(n), np.int32)
    rerr = np.zeros(tuple(n)); pc = np.zeros(3)
    lib.ref_arc_run(_p(b, f64), _p(nn, i32), rcmin, rcmax, rcstep, _p(r, f64), prec, nrefine, _p(err, f64),
                    _p(rcut, f64), _p(idx, i32), _p(rerr, f64), _p(pc, f64))
    return dict(error=err, rcut=rcut, index=idx, result_error=rerr, pcorr=pc)


def ref_fcorr(box, n, rc, rho):
    """The reference's own ForceCorr (oracle/_ref/libref_fcorr.so): reinit(rc, dp) +
    calError(dp); the complex field error2r{x,y,z} (3, nx, ny, nz)."""
    lib = C.CDLL(os.path.join(REF_DIR, "libref_fcorr.so"))
    lib.ref_fcorr_run.argtypes = [P(f64), P(i32), f64, P(f64), P(f64), P(f64)]
    b = np.ascontiguousarray(box, np.float64)
    nn = np.ascontiguousarray(n, np.int32)
    r = np.ascontiguousarray(rho, np.float64).reshape(tuple(n))
    re = np.zeros((3,) + tuple(n)); im = np.zeros((3,) + tuple(n))
    lib.ref_fcorr_run(_p(b, f64), _p(nn, i32), float(rc), _p(r, f64), _p(re, f64), _p(im, f64))
    return re + 1j * im


def ref_spme(pos, q, box, beta, K, rcut, method, order):
    """The reference's own ElectrostaticInteraction (oracle/_ref/libref_spme.so):
    method 0 ik B-spline SPME, 1 analytic-differentiation SPME, 2 exact Ewald."""
    lib = C.CDLL(os.path.join(REF_DIR, "libref_spme.so"))
    lib.ref_spme_forces.argtypes = [i32, P(f64), P(f64), P(f64), f64, P(i32), f64, i32, i32, P(f64), P(f64),
                                    P(f64), P(f64), P(f64), P(f64)]
    p = np.ascontiguousarray(pos, np.float64)
    n = p.shape[0]
    qq = np.ascontiguousarray(q, np.float64)
    b = np.ascontiguousarray(box, np.float64)
    KK = np.ascontiguousarray(K, np.int32)
    df = np.zeros((n, 3)); rf = np.zeros((n, 3))
    e, ed, er, ei = f64(), f64(), f64(), f64()
    lib.ref_spme_forces(n, _p(p, f64), _p(qq, f64), _p(b, f64), beta, _p(KK, i32), rcut, method, order,
                        _p(df, f64), _p(rf, f64), C.byref(e), C.byref(ed), C.byref(er), C.byref(ei))
    return dict(dir=df, rec=rf, energy=e.value, err_dir=ed.value, err_rec=er.value, err_interp=ei.value)


def ref_selfcorr(pos, q, box, beta, K, order):
    """The reference's own SelfCorr (oracle/_ref/libref_spme.so): the self-force
    correction added to zero forces."""
    lib = C.CDLL(os.path.join(REF_DIR, "libref_spme.so"))
    lib.ref_selfcorr.argtypes = [i32, P(f64), P(f64), P(f64), f64, P(i32), i32, P(f64)]
    p = np.ascontiguousarray(pos, np.float64)
    qq = np.ascontiguousarray(q, np.float64)
    b = np.ascontiguousarray(box, np.float64)
    KK = np.ascontiguousarray(K, np.int32)
    F = np.zeros_like(p)
    lib.ref_selfcorr(p.shape[0], _p(p, f64), _p(qq, f64), _p(b, f64), beta, _p(KK, i32), order, _p(F, f64))
    return F


def spme_ik_errmap(K, box, beta, order, rho1, rho2, charge=1.0):
    """Oracle restatement of ErrorEstimate_SPME_Ik::calError on the grid K:
    returns (error1 [K..., 2], error2 [K..., 2]) -- real and imaginary parts."""
    KK = np.ascontiguousarray(K, np.int32)
    b = np.ascontiguousarray(box, np.float64)
    r1 = np.ascontiguousarray(rho1, np.float64).reshape(-1)
    r2 = np.ascontiguousarray(rho2, np.float64).reshape(-1)
    n = int(np.prod(K))
    e1 = np.zeros(2 * n)
    e2 = np.zeros(2 * n)
    _lib.orc_spme_ik_errmap(_p(KK, i32), _p(b, f64), float(beta), int(order), _p(r1, f64), _p(r2, f64),
                            float(charge), _p(e1, f64), _p(e2, f64))
    return e1.reshape(tuple(K) + (2,)), e2.reshape(tuple(K) + (2,))


def dir_errmap(K, box, beta, rcut, rho1, rho2, charge=1.0):
    """ErrorEstimate_dir::reinit + calError restated (oracle_errmap.c): error1, error2 as
    (K0, K1, K2, 2) arrays (real, imaginary)."""
    KK = np.ascontiguousarray(K, np.int32)
    b = np.ascontiguousarray(box, np.float64)
    r1 = np.ascontiguousarray(rho1, np.float64).reshape(tuple(K))
    r2 = np.ascontiguousarray(rho2, np.float64).reshape(tuple(K))
    e1 = np.zeros(tuple(K) + (2,)); e2 = np.zeros(tuple(K) + (2,))
    _lib.orc_dir_errmap(_p(KK, i32), _p(b, f64), float(beta), float(rcut), _p(r1, f64), _p(r2, f64),
                        float(charge), _p(e1, f64), _p(e2, f64))
    return e1, e2


def ref_dir_errmap(K, box, beta, rcut, rho1, rho2, charge=1.0):
    """The reference's own ErrorEstimate_dir (oracle/_ref/libref_errdir.so)."""
    lib = C.CDLL(os.path.join(REF_DIR, "libref_errdir.so"))
    lib.ref_dir_errmap.argtypes = [P(i32), P(f64), f64, f64, P(f64), P(f64), f64, P(f64), P(f64)]
    KK = np.ascontiguousarray(K, np.int32)
    b = np.ascontiguousarray(box, np.float64)
    r1 = np.ascontiguousarray(rho1, np.float64).reshape(tuple(K))
    r2 = np.ascontiguousarray(rho2, np.float64).reshape(tuple(K))
    e1 = np.zeros(tuple(K) + (2,)); e2 = np.zeros(tuple(K) + (2,))
    lib.ref_dir_errmap(_p(KK, i32), _p(b, f64), float(beta), float(rcut), _p(r1, f64), _p(r2, f64),
                       float(charge), _p(e1, f64), _p(e2, f64))
    return e1, e2


def ref_spme_ik_errmap(K, box, beta, order, rho1, rho2, charge=1.0):
    """The reference's own ErrorEstimate_SPME_Ik (oracle/_ref/libref_errmap.so)."""
    lib = C.CDLL(os.path.join(REF_DIR, "libref_errmap.so"))
    lib.ref_spme_ik_errmap.argtypes = [P(i32), P(f64), f64, i32, P(f64), P(f64), f64, P(f64), P(f64)]
    KK = np.ascontiguousarray(K, np.int32)
    b = np.ascontiguousarray(box, np.float64)
    r1 = np.ascontiguousarray(rho1, np.float64).reshape(-1)
    r2 = np.ascontiguousarray(rho2, np.float64).reshape(-1)
    n = int(np.prod(K))
    e1 = np.zeros(2 * n)
    e2 = np.zeros(2 * n)
    lib.ref_spme_ik_errmap(_p(KK, i32), _p(b, f64), float(beta), int(order), _p(r1, f64), _p(r2, f64),
                           float(charge), _p(e1, f64), _p(e2, f64))
    return e1.reshape(tuple(K) + (2,)), e2.reshape(tuple(K) + (2,))


def dft3d(data, sign):
    """The oracle's unnormalised 3D DFT (sign -1 forward, +1 backward)."""
    a = np.ascontiguousarray(data, np.complex128)
    n = np.ascontiguousarray(a.shape, np.int32)
    buf = np.ascontiguousarray(np.stack([a.real, a.imag], -1), np.float64)
    _lib.orc_dft3d(_p(n, i32), _p(buf, f64), int(sign))
    return buf[..., 0] + 1j * buf[..., 1]


def spme_selfcorr(pos, q, box, K, order, beta):
    """Oracle restatement of SelfCorr: the correction added to zero forces."""
    p = np.ascontiguousarray(pos, np.float64)
    qq = np.ascontiguousarray(q, np.float64)
    b = np.ascontiguousarray(box, np.float64)
    KK = np.ascontiguousarray(K, np.int32)
    F = np.zeros_like(p)
    _lib.orc_spme_selfcorr(p.shape[0], _p(p, f64), _p(qq, f64), _p(b, f64), _p(KK, i32), order, beta, _p(F, f64))
    return F


# ---------------------------------------------------------------- SPME / Ewald
_sigs3 = {
    "orc_bspline_weights": (None, [i32, f64, P(f64), P(f64)]),
    "orc_bspline": (f64, [i32, f64]),
    "orc_spme_bmod": (None, [i32, i32, P(f64)]),
    "orc_spme_spread": (None, [i32, P(f64), P(f64), P(f64), P(i32), i32, P(f64)]),
    "orc_spme_rec": (f64, [i32, P(f64), P(f64), P(f64), P(i32), i32, f64, i32, P(f64)]),
    "orc_ewald_rec_exact": (f64, [i32, P(f64), P(f64), P(f64), P(i32), f64, P(f64)]),
    "orc_ewald_dir": (f64, [i32, P(f64), P(f64), P(f64), f64, f64, P(f64)]),
    "orc_ewald_self": (f64, [i32, P(f64), f64]),
    "orc_spme_selfcorr": (None, [i32, P(f64), P(f64), P(f64), P(i32), i32, f64, P(f64)]),
    "orc_spme_ik_errmap": (None, [P(i32), P(f64), f64, i32, P(f64), P(f64), f64, P(f64), P(f64)]),
    "orc_dir_errmap": (None, [P(i32), P(f64), f64, f64, P(f64), P(f64), f64, P(f64), P(f64)]),
    "orc_lj_allpair_typed": (None, [i32, P(f64), P(f64), P(i32), i32, P(f64), P(i32), P(f64), P(f32), P(f32),
                                    P(f64), P(f64)]),
    "orc_nb_pair": (None, [i32, P(f64), i32, P(f64), P(f64), P(f64)]),
    "orc_bond_term": (None, [i32, P(f64), i32, P(f64), P(f64), P(f64)]),
    "orc_angle_term": (None, [i32, P(f64), i32, P(f64), P(f64), P(f64), P(f64), P(f64)]),
    "orc_bonded_apply": (None, [i32, P(f64), P(f64), i32, i32, P(i32), P(i32), P(f64), i32, P(i32), P(i32),
                                P(f64), P(f64), P(f64)]),
    "orc_spme_ana_errmap": (None, [P(i32), P(f64), f64, i32, P(f64), P(f64), f64, P(f64), P(f64),
                                   P(f64), P(f64)]),
    "orc_dft3d": (None, [P(i32), P(f64), i32]),
}
for _n, (_r, _a) in _sigs3.items():
    _f = getattr(_lib, _n)
    _f.restype = _r
    _f.argtypes = _a


def bspline_weights(n, f):
    w = np.zeros(n); dw = np.zeros(n)
    _lib.orc_bspline_weights(n, float(f), _p(w, f64), _p(dw, f64))
    return w, dw


def bspline(n, x):
    return _lib.orc_bspline(n, float(x))


def spme_bmod(n, K):
    b = np.zeros(K)
    _lib.orc_spme_bmod(n, K, _p(b, f64))
    return b


def spme_spread(pos, q, box, K, n):
    p = np.ascontiguousarray(pos, np.float64); qq = np.ascontiguousarray(q, np.float64)
    b = np.ascontiguousarray(box, np.float64); KK = np.ascontiguousarray(K, np.int32)
    Q = np.zeros(tuple(K))
    _lib.orc_spme_spread(p.shape[0], _p(p, f64), _p(qq, f64), _p(b, f64), _p(KK, i32), n, _p(Q, f64))
    return Q


def spme_rec(pos, q, box, K, n, beta, method=0):
    """reciprocal SPME energy and forces; method 0 ik, 1 analytic differentiation"""
    p = np.ascontiguousarray(pos, np.float64); qq = np.ascontiguousarray(q, np.float64)
    b = np.ascontiguousarray(box, np.float64); KK = np.ascontiguousarray(K, np.int32)
    F = np.zeros_like(p)
    E = _lib.orc_spme_rec(p.shape[0], _p(p, f64), _p(qq, f64), _p(b, f64), _p(KK, i32), n, beta, method, _p(F, f64))
    return E, F


def ewald_rec_exact(pos, q, box, K, beta):
    p = np.ascontiguousarray(pos, np.float64); qq = np.ascontiguousarray(q, np.float64)
    b = np.ascontiguousarray(box, np.float64); KK = np.ascontiguousarray(K, np.int32)
    F = np.zeros_like(p)
    E = _lib.orc_ewald_rec_exact(p.shape[0], _p(p, f64), _p(qq, f64), _p(b, f64), _p(KK, i32), beta, _p(F, f64))
    return E, F


def ewald_dir(pos, q, box, beta, rcut):
    p = np.ascontiguousarray(pos, np.float64); qq = np.ascontiguousarray(q, np.float64)
    b = np.ascontiguousarray(box, np.float64)
    F = np.zeros_like(p)
    E = _lib.orc_ewald_dir(p.shape[0], _p(p, f64), _p(qq, f64), _p(b, f64), beta, rcut, _p(F, f64))
    return E, F


def ewald_self(q, beta):
    qq = np.ascontiguousarray(q, np.float64)
    return _lib.orc_ewald_self(len(qq), _p(qq, f64), beta)


# ---------------------------------------------------------------- error estimates
_lib.orc_error_estimate_pme.restype = None
_lib.orc_error_estimate_pme.argtypes = [P(f64), P(i32), f64, f64, f64, i32, P(f64), P(f64)]
_lib.orc_error_estimate_spme_ik.restype = f64
_lib.orc_error_estimate_spme_ik.argtypes = [P(f64), P(i32), i32, f64, f64, i32]


def error_estimate_pme(box, K, beta, rcut, c2, natom):
    b = np.ascontiguousarray(box, np.float64); KK = np.ascontiguousarray(K, np.int32)
    d, r = f64(), f64()
    _lib.orc_error_estimate_pme(_p(b, f64), _p(KK, i32), beta, rcut, c2, natom, C.byref(d), C.byref(r))
    return d.value, r.value


def error_estimate_spme_ik(box, K, order, beta, c2, natom):
    b = np.ascontiguousarray(box, np.float64); KK = np.ascontiguousarray(K, np.int32)
    return _lib.orc_error_estimate_spme_ik(_p(b, f64), _p(KK, i32), order, beta, c2, natom)


def ref_gro_read(path, n):
    """The reference engine's own GromacsFileManager::readGroFile
    (oracle/_ref/libref_gro.so): binary32 values; None when it threw."""
    lib = C.CDLL(os.path.join(REF_DIR, "libref_gro.so"))
    lib.ref_gro_read.argtypes = [C.c_char_p, i32, P(i32), P(C.c_char), P(C.c_char), P(i32), P(C.c_float),
                                 P(C.c_float), P(C.c_float)]
    ri = np.zeros(n, np.int32); ai = np.zeros(n, np.int32)
    rn = np.zeros((n, 8), np.uint8); an = np.zeros((n, 8), np.uint8)
    pos = np.zeros((n, 3), np.float32); vel = np.zeros((n, 3), np.float32); box = np.zeros(3, np.float32)
    r = lib.ref_gro_read(str(path).encode(), n, _p(ri, i32), _p(rn, C.c_char), _p(an, C.c_char), _p(ai, i32),
                         _p(pos, C.c_float), _p(vel, C.c_float), _p(box, C.c_float))
    if r:
        return None
    dec = lambda row: bytes(row).split(b"\0", 1)[0].decode()
    return dict(resd_index=ri, atom_index=ai, resd_name=[dec(x) for x in rn], atom_name=[dec(x) for x in an],
                pos=pos, vel=vel, box=box)


def ref_gro_write(path, title, resd_index, resd_name, atom_name, atom_index, pos, vel, box):
    """The reference engine's GromacsFileManager::writeGroFile after `title`, from binary32 arrays."""
    lib = C.CDLL(os.path.join(REF_DIR, "libref_gro.so"))
    lib.ref_gro_write.argtypes = [C.c_char_p, C.c_char_p, i32, P(i32), P(C.c_char), P(C.c_char), P(i32),
                                  P(C.c_float), P(C.c_float), P(C.c_float)]
    n = len(resd_index)
    slots = lambda names: np.array([list(s.encode()[:7].ljust(8, b"\0")) for s in names], np.uint8).reshape(n, 8)
    rn, an = slots(resd_name), slots(atom_name)
    ri = np.ascontiguousarray(resd_index, np.int32); ai = np.ascontiguousarray(atom_index, np.int32)
    p = np.ascontiguousarray(pos, np.float32); v = np.ascontiguousarray(vel, np.float32)
    b = np.ascontiguousarray(box, np.float32)
    return lib.ref_gro_write(str(path).encode(), title.encode(), n, _p(ri, i32), _p(rn, C.c_char), _p(an, C.c_char),
                             _p(ai, i32), _p(p, C.c_float), _p(v, C.c_float), _p(b, C.c_float))


def bond_term(btype, uparam, prec, d):
    """Force on the reference atom and energy of one bond term (oracle_bonded.c)."""
    u = np.zeros(3); u[:len(uparam)] = uparam
    dd = np.ascontiguousarray(d, np.float64); f = np.zeros(3); e = C.c_double()
    _lib.orc_bond_term(int(btype), _p(u, f64), int(prec), _p(dd, f64), _p(f, f64), C.byref(e))
    return f, e.value


def angle_term(atype, uparam, prec, d0, d1):
    """forcePoten01 of one angle term (oracle_bonded.c): f0, f1, energy."""
    u = np.zeros(3); u[:len(uparam)] = uparam
    a = np.ascontiguousarray(d0, np.float64); b = np.ascontiguousarray(d1, np.float64)
    f0 = np.zeros(3); f1 = np.zeros(3); e = C.c_double()
    _lib.orc_angle_term(int(atype), _p(u, f64), int(prec), _p(a, f64), _p(b, f64), _p(f0, f64), _p(f1, f64),
                        C.byref(e))
    return f0, f1, e.value


def bonded_apply(pos, box, prec, bonds, btype, bparam, angles, atype, aparam):
    """The engine's per-atom bonded gather (oracle_bonded.c): forces [n, 3] in
    original order and (energy, virial xx, yy, zz)."""
    p = np.ascontiguousarray(pos, np.float64); b = np.ascontiguousarray(box, np.float64)
    n = p.shape[0]
    bo = np.ascontiguousarray(bonds, np.int32).reshape(-1, 2); bt = np.ascontiguousarray(btype, np.int32)
    bp = np.zeros((len(bo), 3)); bp[:, :np.shape(bparam)[1] if len(bo) else 0] = bparam if len(bo) else 0
    an = np.ascontiguousarray(angles, np.int32).reshape(-1, 3); at = np.ascontiguousarray(atype, np.int32)
    ap = np.zeros((len(an), 3)); ap[:, :np.shape(aparam)[1] if len(an) else 0] = aparam if len(an) else 0
    f = np.zeros((n, 3)); st = np.zeros(4)
    _lib.orc_bonded_apply(n, _p(p, f64), _p(b, f64), int(prec), len(bo), _p(bo, i32), _p(bt, i32), _p(bp, f64),
                          len(an), _p(an, i32), _p(at, i32), _p(ap, f64), _p(f, f64), _p(st, f64))
    return f, st


def ref_bonded_term(ftype, uparam, d0, d1=None):
    """The reference's own bond / angle force functions (oracle/_ref/libref_bonded.so,
    binary32): bond -> (f, e); angle (forcePoten01) -> (f0, f1, e)."""
    lib = C.CDLL(os.path.join(REF_DIR, "libref_bonded.so"))
    lib.ref_bonded_term.argtypes = [i32, P(f64), P(f64), P(f64), P(f64), P(f64), P(f64)]
    u = np.zeros(3); u[:len(uparam)] = uparam
    a = np.ascontiguousarray(d0, np.float64)
    b = np.zeros(3) if d1 is None else np.ascontiguousarray(d1, np.float64)
    f0 = np.zeros(3); f1 = np.zeros(3); e = np.zeros(1)
    lib.ref_bonded_term(int(ftype), _p(u, f64), _p(a, f64), _p(b, f64), _p(f0, f64), _p(f1, f64), _p(e, f64))
    return (f0, float(e[0])) if d1 is None else (f0, f1, float(e[0]))


def nb_pair(kind, uparam, prec, d):
    """One non-bonded pair of a kind (oracle_md.c): force on i, energy."""
    u = np.zeros(6); u[:len(uparam)] = uparam
    dd = np.ascontiguousarray(d, np.float64); f = np.zeros(3); e = C.c_double()
    _lib.orc_nb_pair(int(kind), _p(u, f64), int(prec), _p(dd, f64), _p(f, f64), C.byref(e))
    return f, e.value


def ref_nb_pair(kind, uparam, d):
    """The reference's own pair functions (oracle/_ref/libref_nb.so), binary32."""
    lib = C.CDLL(os.path.join(REF_DIR, "libref_nb.so"))
    lib.ref_nb_pair.argtypes = [i32, P(f64), P(f64), P(f64), P(f64)]
    u = np.zeros(6); u[:len(uparam)] = uparam
    dd = np.ascontiguousarray(d, np.float64); f = np.zeros(3); e = np.zeros(1)
    lib.ref_nb_pair(int(kind), _p(u, f64), _p(dd, f64), _p(f, f64), _p(e, f64))
    return f, float(e[0])
