"""Host-side mirror of the md.error interaction-engine API over the C ABI.

Class and method names follow the reference engine
(shortRange.inhomo/template/tools/simulation.hetero.cutoff):
  MDSystem            include/MDSystem_interface.h:18-104
  CellList            include/CellList_interface.h:18-73 (rebuild)
  NeighborList        include/NeighborList_interface.h:20-82 (rebuild)
  InteractionEngine   include/InteractionEngine_interface.h:17-155
                      (registNonBondedInteraction, clearInteraction,
                       applyNonBondedInteraction, applyBondedInteraction)
  AssignRCut          include/AssignRCut.h:10-42 (getRCut + assign)
  VelocityVerlet      include/Integrator_interface.h:181-205 (step1/step2)
Errors are raised as MDException subclasses named after the reference's
exceptions / device flags (MDExcptCuda, mdErrorShortNeighborList, ...).
"""
import ctypes as C

import numpy as np

from ._lib import lib, LangevinParams, SimParams

MD_OK = 0
MD_ERR_CELL_OVERFLOW = 1
MD_ERR_NLIST_OVERFLOW = 2
MD_ERR_CELL_INDEX = 3
MD_ERR_CUDA = 10
MD_ERR_BADARG = 11
MD_ERR_UNSUPPORTED = 12
MD_ERR_TIMEOUT = 13
MD_ERR_NOMEM = 14
MD_ERR_IO = 15

PREC_MIXED = 0
PREC_FP64 = 1
INTEG_LANGEVIN = 0
INTEG_NHC = 1
NL_MINIMAGE = 0
NL_CELLSHIFT = 1

STAT_NB_ENERGY, STAT_VIRIAL_XX, STAT_VIRIAL_YY, STAT_VIRIAL_ZZ = 0, 1, 2, 3
STAT_ELEC_DIR = 4
STAT_KINETIC_XX, STAT_KINETIC_YY, STAT_KINETIC_ZZ = 5, 6, 7
STAT_PRESSURE_CORR_XX = 8
STAT_ELEC_REC, STAT_ELEC_SELF = 11, 12
STAT_BOND_ENERGY = 13
BOND_HARMONIC, BOND_FENE, BOND_FENE2 = 10000, 10001, 10002
NB_NULL, NB_LJ6_12, NB_LJ6_12_CAP, NB_COSTAIL, NB_COSTAIL_CAP, NB_LJ6_12B, NB_LJ6_12B_CAP = 0, 1, 2, 3, 4, 5, 6
ANGLE_HARMONIC, ANGLE_COS0 = 20000, 20001
STAT_COUNT = 16

# cudaStreamLegacy (cuda_runtime_api.h): the legacy default stream as an explicit handle
CUDA_STREAM_LEGACY = 0x1


class MDException(RuntimeError):
    code = -1


class MDExcptCuda(MDException):
    code = MD_ERR_CUDA


class MDExcptShortCellList(MDException):
    code = MD_ERR_CELL_OVERFLOW


class MDExcptShortNeighborList(MDException):
    code = MD_ERR_NLIST_OVERFLOW


class MDExcptCellIndexOverflow(MDException):
    code = MD_ERR_CELL_INDEX


class MDExcptBadArgument(MDException, ValueError):
    code = MD_ERR_BADARG


class MDExcptUnsupported(MDException):
    code = MD_ERR_UNSUPPORTED


class MDExcptTimeout(MDException):
    code = MD_ERR_TIMEOUT


class MDExcptIO(MDException, OSError):
    """MDExcptCannotOpenFile / MDExcptWrongFileFormat of the reference."""
    code = MD_ERR_IO


_BY_CODE = {c.code: c for c in (MDExcptCuda, MDExcptShortCellList, MDExcptShortNeighborList,
                                 MDExcptCellIndexOverflow, MDExcptBadArgument,
                                 MDExcptUnsupported, MDExcptTimeout, MDExcptIO)}


def check(status, what=""):
    if status != MD_OK:
        msg = lib.md_last_error_message().decode()
        raise _BY_CODE.get(status, MDException)(f"{what}: {msg} (status {status})")


def _p(a, ctype=C.c_double):
    return a.ctypes.data_as(C.POINTER(ctype))


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


def device_count():
    n = C.c_int(0)
    check(lib.md_device_count(C.byref(n)), "md_device_count")
    return n.value


class MDSystem:
    """Per-atom SoA on the device (MDSystem / DeviceMDData)."""

    def __init__(self, pos, box, vel=None, charge=None, mass=None, precision=PREC_MIXED, device=0, type=None):
        pos = _f64(pos).reshape(-1, 3)
        self.n = pos.shape[0]
        box = _f64(box, (3,))
        self.precision = precision
        h = C.c_void_p()
        args = [C.byref(h), self.n, _p(box), _p(pos)]
        keep = []
        for arr, shape in ((vel, (-1, 3)),):
            if arr is None:
                args.append(None)
            else:
                a = _f64(arr).reshape(shape)
                keep.append(a)
                args.append(_p(a))
        if type is None:
            args.append(None)
        else:
            t = np.ascontiguousarray(type, np.int32).reshape(-1)
            keep.append(t)
            args.append(_p(t, C.c_int))
        for arr in (charge, mass):
            if arr is None:
                args.append(None)
            else:
                a = _f64(arr).reshape(-1)
                keep.append(a)
                args.append(_p(a))
        args += [precision, device]
        check(lib.md_system_create(*args), "MDSystem")
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            lib.md_system_destroy(self.h)
            self.h = None

    def set_stream(self, stream_ptr):
        """Issue the system's device work on the CUDA stream with this handle
        (e.g. torch's `Stream.cuda_stream`).  0, the handle torch gives its
        default stream, means the legacy default stream and is passed as
        cudaStreamLegacy, since a NULL handle selects the library's own
        stream; None goes back to the library's own stream."""
        if stream_ptr is None:
            h = None
        elif int(stream_ptr) == 0:
            h = CUDA_STREAM_LEGACY
        else:
            h = int(stream_ptr)
        check(lib.md_system_set_stream(self.h, C.c_void_p(h)), "set_stream")

    def synchronize(self):
        check(lib.md_system_synchronize(self.h), "synchronize")

    def set_types(self, type):
        """Atom types 0..15 in original order (MDSystem hdata.type)."""
        t = np.ascontiguousarray(type, np.int32).reshape(-1)
        check(lib.md_system_set_types(self.h, _p(t, C.c_int)), "set_types")

    def types(self):
        out = np.empty(self.n, np.int32)
        check(lib.md_system_get_types(self.h, _p(out, C.c_int)), "types")
        return out

    def _get3(self, fn):
        out = np.empty((self.n, 3), np.float64)
        check(fn(self.h, _p(out)), fn.__name__)
        return out

    def positions(self):
        return self._get3(lib.md_system_get_positions)

    def unwrapped_positions(self):
        return self._get3(lib.md_system_get_unwrapped_positions)

    def velocities(self):
        return self._get3(lib.md_system_get_velocities)

    def forces(self):
        return self._get3(lib.md_system_get_forces)

    def set_positions(self, pos):
        a = _f64(pos).reshape(self.n, 3)
        check(lib.md_system_set_positions(self.h, _p(a)), "set_positions")

    def set_velocities(self, vel):
        a = _f64(vel).reshape(self.n, 3)
        check(lib.md_system_set_velocities(self.h, _p(a)), "set_velocities")

    def charges(self):
        q = np.empty(self.n, np.float64)
        check(lib.md_system_get_charges(self.h, _p(q)), "get_charges")
        return q

    def set_charges(self, q):
        a = _f64(q).reshape(self.n)
        check(lib.md_system_set_charges(self.h, _p(a)), "set_charges")

    def set_device_view(self, pos_ptr=None, charge_ptr=None):
        """Positions [N,3] and/or charges [N] from device memory (raw pointers, e.g.
        torch tensors' data_ptr(), caller's atom order), without a host copy
        (md_system_set_device_view).  Asynchronous on the system's stream."""
        from ._lib import DeviceView
        v = DeviceView(pos_ptr or None, charge_ptr or None)
        check(lib.md_system_set_device_view(self.h, C.byref(v)), "set_device_view")

    def set_masses(self, m):
        """Per-atom masses in original order (MDSystem hdata.mass)."""
        a = _f64(m).reshape(self.n)
        check(lib.md_system_set_masses(self.h, _p(a)), "set_masses")

    def masses(self):
        out = np.empty(self.n, np.float64)
        check(lib.md_system_get_masses(self.h, _p(out)), "masses")
        return out

    def box(self):
        b = np.empty(3, np.float64)
        check(lib.md_system_get_box(self.h, _p(b)), "get_box")
        return b

    def set_box(self, box):
        b = _f64(box, (3,))
        check(lib.md_system_set_box(self.h, _p(b)), "set_box")

    def set_rcut(self, rcut):
        a = np.ascontiguousarray(rcut, dtype=np.float32).reshape(self.n)
        check(lib.md_system_set_rcut(self.h, _p(a, C.c_float)), "set_rcut")

    def rcut(self):
        a = np.empty(self.n, np.float32)
        check(lib.md_system_get_rcut(self.h, _p(a, C.c_float)), "get_rcut")
        return a

    def normalizeDeviceData(self):
        check(lib.md_system_normalize(self.h), "normalize")

    def stats(self):
        out = np.zeros(STAT_COUNT, np.float64)
        check(lib.md_system_read_stats(self.h, _p(out)), "read_stats")
        return out

    def stats_async(self, out):
        """Queue a copy of the statistic slots into out (float64, MD_STAT_COUNT,
        page-locked for a copy that does not wait); out is valid after
        synchronize()."""
        if out.dtype != np.float64 or out.size < STAT_COUNT or not out.flags.c_contiguous:
            raise ValueError("stats_async: out must be a contiguous float64 array of STAT_COUNT entries")
        check(lib.md_system_read_stats_async(self.h, _p(out)), "read_stats_async")

    def clear_stats(self):
        check(lib.md_system_clear_stats(self.h), "clear_stats")

    def pressure(self, stats=None):
        """MDStatistic::pressureXX/YY/ZZ (ENG/include/Statistic_interface.h:92-121)."""
        s = self.stats() if stats is None else stats
        L = self.box()
        V = L.prod()
        return np.array([2.0 / V * (s[STAT_KINETIC_XX + d] - 0.5 * s[STAT_VIRIAL_XX + d])
                         + s[STAT_PRESSURE_CORR_XX + d] for d in range(3)])


class CellList:
    def __init__(self, sys, cell_size, bdir=7, divide=1):
        h = C.c_void_p()
        check(lib.md_cell_list_create(C.byref(h), sys.h, float(cell_size), bdir, divide), "CellList")
        self.h = h
        self.sys = sys

    def __del__(self):
        if getattr(self, "h", None):
            lib.md_cell_list_destroy(self.h)
            self.h = None

    def rebuild(self, sys=None):
        check(lib.md_cell_list_rebuild(self.h, (sys or self.sys).h), "CellList::rebuild")

    def ncell(self):
        a = (C.c_int * 3)()
        check(lib.md_cell_list_get_ncell(self.h, a), "ncell")
        return tuple(a)

    def cell_index(self):
        out = np.empty(self.sys.n, np.uint32)
        check(lib.md_cell_list_get_cell_index(self.h, self.sys.h, _p(out, C.c_uint32)), "cell_index")
        return out


class NeighborList:
    def __init__(self, sys, rlist, skin, expansion=4.0, mode=NL_MINIMAGE):
        h = C.c_void_p()
        check(lib.md_nlist_create(C.byref(h), sys.h, float(rlist), float(skin), float(expansion), mode),
              "NeighborList")
        self.h = h
        self.sys = sys

    def __del__(self):
        if getattr(self, "h", None):
            lib.md_nlist_destroy(self.h)
            self.h = None

    def rebuild(self, sys, clist):
        check(lib.md_nlist_rebuild(self.h, sys.h, clist.h), "NeighborList::rebuild")

    def fit(self, sys, clist):
        check(lib.md_nlist_fit(self.h, sys.h, clist.h), "NeighborList::fit")

    def capacity(self):
        c = C.c_int()
        check(lib.md_nlist_capacity(self.h, C.byref(c)), "capacity")
        return c.value

    def calSumNeighbor(self):
        s = C.c_int64()
        check(lib.md_nlist_sum_neighbor(self.h, self.sys.h, C.byref(s)), "calSumNeighbor")
        return s.value

    def max_displacement(self):
        d = C.c_double()
        check(lib.md_nlist_max_displacement(self.h, self.sys.h, C.byref(d)), "max_displacement")
        return d.value

    def lists(self):
        """(counts[N], pairs) in original atom indices (CSR order)."""
        counts = np.empty(self.sys.n, np.int32)
        total = self.calSumNeighbor()
        pairs = np.empty(max(total, 1), np.int32)
        check(lib.md_nlist_get(self.h, self.sys.h, _p(counts, C.c_int32), _p(pairs, C.c_int32)), "nlist_get")
        return counts, pairs[:total]


class InteractionEngine:
    def __init__(self, sys):
        h = C.c_void_p()
        check(lib.md_engine_create(C.byref(h), sys.h), "InteractionEngine")
        self.h = h
        self.sys = sys

    def __del__(self):
        if getattr(self, "h", None):
            lib.md_engine_destroy(self.h)
            self.h = None

    def registNonBondedInteraction(self, epsilon=1.0, sigma=1.0, shift=0.0):
        check(lib.md_engine_register_lj(self.h, epsilon, sigma, shift), "registNonBondedInteraction")

    def registNonBondedInteractionPair(self, type0, type1, epsilon=1.0, sigma=1.0, shift=0.0):
        """SystemNonBondedInteraction::add(type0, type1, LennardJones6_12Parameter):
        LJ for one pair of atom types; pairs never given take no force."""
        check(lib.md_engine_register_lj_pair(self.h, int(type0), int(type1), float(epsilon), float(sigma),
                                             float(shift)), "registNonBondedInteractionPair")

    def registNonBondedPair(self, type0, type1, kind, params):
        """A pair kind of the nbForce dispatch for a type pair: NB_LJ6_12 (eps, sigma,
        shift), NB_LJ6_12B (eps, sigma, shift, rcut), NB_LJ6_12_CAP / NB_LJ6_12B_CAP
        (eps, sigma, shift, rcut, cap), NB_COSTAIL (eps, b, wc), NB_COSTAIL_CAP
        (eps, b, wc, cap), NB_NULL."""
        q = np.zeros(6)
        q[:len(params)] = params
        check(lib.md_engine_register_nb_pair(self.h, int(type0), int(type1), int(kind), _p(q)),
              "registNonBondedPair")

    def setForceCorrection(self, fc):
        """the non-bonded kernel adds the per-atom LFC values (None: off)"""
        check(lib.md_engine_set_force_correction(self.h, fc.h if fc is not None else None), "setForceCorrection")
        self.fcorr = fc

    def registBondedInteraction(self, n_bonds=0):
        check(lib.md_engine_register_bonded(self.h, int(n_bonds)), "registBondedInteraction")

    @staticmethod
    def _terms(atoms, types, params, width):
        a = np.ascontiguousarray(atoms, np.int32).reshape(-1, width)
        n = a.shape[0]
        t = np.ascontiguousarray(np.broadcast_to(np.asarray(types, np.int32), (n,)))
        p = np.zeros((n, 3))
        if n:
            q = np.asarray(params, np.float64)
            q = np.broadcast_to(q, (n,) + q.shape[-1:]) if q.ndim == 1 else q.reshape(n, -1)
            p[:, :q.shape[1]] = q
        return a, t, p

    def setBonds(self, atoms, types, params):
        """Bonds [n, 2] (original atom order), types BOND_* and parameters as the
        reference's HarmonicSpringParameter(k, r0) / FENEParameter(k, rinf) /
        FENE2Parameter(k, rs, r0) take them ([n, <=3] or one row for all)."""
        a, t, p = self._terms(atoms, types, params, 2)
        check(lib.md_engine_set_bonds(self.h, a.shape[0], _p(a, C.c_int), _p(t, C.c_int), _p(p)), "setBonds")
        self._bonds = (a, t, p)

    def setAngles(self, atoms, types, params):
        """Angles [n, 3] (edge0, centre, edge1), types ANGLE_* and parameters
        AngleHarmonicParameter(k, theta0) / CosAngle0Parameter(k)."""
        a, t, p = self._terms(atoms, types, params, 3)
        check(lib.md_engine_set_angles(self.h, a.shape[0], _p(a, C.c_int), _p(t, C.c_int), _p(p)), "setAngles")
        self._angles = (a, t, p)

    def setExclusions(self, pairs):
        """Pairs [n, 2] that take no non-bonded force (ExclusionList)."""
        a = np.ascontiguousarray(pairs, np.int32).reshape(-1, 2)
        check(lib.md_engine_set_exclusions(self.h, a.shape[0], _p(a, C.c_int)), "setExclusions")

    def clearInteraction(self, sys=None):
        check(lib.md_engine_clear_forces(self.h, (sys or self.sys).h), "clearInteraction")

    def applyNonBondedInteraction(self, sys, nlist, with_stats=True):
        """with_stats True / False, or "rows": the force kernel as the step
        driver runs it, its statistics left as per-warp rows for
        finishNonBondedStatistics."""
        mode = 2 if with_stats == "rows" else (1 if with_stats else 0)
        check(lib.md_engine_apply_nonbonded(self.h, sys.h, nlist.h, mode), "applyNonBondedInteraction")

    def finishNonBondedStatistics(self, sys):
        check(lib.md_engine_finish_nonbonded_stats(self.h, sys.h), "finishNonBondedStatistics")

    def applyBondedInteraction(self, sys):
        check(lib.md_engine_apply_bonded(self.h, sys.h), "applyBondedInteraction")


def registCoulomb(engine, beta):
    """Real-space Ewald in the non-bonded kernel (ElectrostaticInteraction_dir)."""
    check(lib.md_engine_register_coulomb(engine.h, float(beta)), "registCoulomb")


class SPME:
    """Reciprocal SPME on the device: ElectrostaticInteraction_rec_BSpline (method 'ik')
    or ElectrostaticInteraction_rec_FBSpline (method 'analytic')."""

    def __init__(self, sys, K, order, beta, method="ik"):
        KK = (C.c_int * 3)(*[int(k) for k in K])
        h = C.c_void_p()
        m = {"ik": 0, "analytic": 1}[method]
        check(lib.md_spme_create(C.byref(h), sys.h, KK, int(order), float(beta), m), "SPME")
        self.h = h
        self.sys = sys
        self.K = tuple(int(k) for k in K)
        self.beta = beta

    def __del__(self):
        if getattr(self, "h", None):
            lib.md_spme_destroy(self.h)
            self.h = None

    def apply(self, sys=None, with_stats=True):
        check(lib.md_spme_apply(self.h, (sys or self.sys).h, 1 if with_stats else 0), "SPME::apply")

    def mesh(self):
        Q = np.empty(self.K, np.float64)
        check(lib.md_spme_get_mesh(self.h, _p(Q)), "mesh")
        return Q

    def self_correction(self, sys=None):
        """SelfCorr::correction: add the analytic-differentiation self-force correction."""
        check(lib.md_spme_self_correction(self.h, (sys or self.sys).h), "SPME::self_correction")

    def influence(self):
        """psi on the half spectrum [K0, K1, K2/2+1]."""
        psi = np.empty((self.K[0], self.K[1], self.K[2] // 2 + 1), np.float64)
        check(lib.md_spme_get_influence(self.h, _p(psi)), "influence")
        return psi

    def energy_grad_device(self, energy_ptr, dq_ptr=None, dr_ptr=None, dbeta_ptr=None):
        """md_spme_energy_grad with outputs in device memory (raw pointers; energy and
        dE/dbeta one double each, dE/dq [N], dE/dr [N,3]); no host copy, no wait."""
        check(lib.md_spme_energy_grad_device(self.h, self.sys.h, energy_ptr, dq_ptr, dr_ptr, dbeta_ptr),
              "SPME::energy_grad_device")

    def energy_grad(self, dq=True, dr=True, dpsi=False):
        """Reciprocal energy and its exact gradient (md_spme_energy_grad):
        dict with energy, dE_dbeta and, as asked, dE_dq [N], dE_dr [N, 3],
        dE_dpsi [K0, K1, K2/2+1]."""
        n = self.sys.n
        e, db = C.c_double(), C.c_double()
        gq = np.empty(n) if dq else None
        gr = np.empty((n, 3)) if dr else None
        gp = np.empty((self.K[0], self.K[1], self.K[2] // 2 + 1)) if dpsi else None
        check(lib.md_spme_energy_grad(self.h, self.sys.h, C.byref(e), _p(gq) if dq else None,
                                      _p(gr) if dr else None, C.byref(db), _p(gp) if dpsi else None),
              "SPME::energy_grad")
        out = {"energy": e.value, "dE_dbeta": db.value}
        if dq:
            out["dE_dq"] = gq
        if dr:
            out["dE_dr"] = gr
        if dpsi:
            out["dE_dpsi"] = gp
        return out


def ewald_self_energy(sys, beta):
    v = C.c_double()
    check(lib.md_ewald_self_energy(sys.h, float(beta), C.byref(v)), "self energy")
    return v.value


def ewald_exact(sys, K, beta, add_forces=True):
    """Exact reciprocal Ewald sum in FP64 (ElectrostaticInteraction_rec_ES)."""
    KK = (C.c_int * 3)(*[int(k) for k in K])
    e = C.c_double()
    check(lib.md_ewald_exact(sys.h, KK, float(beta), C.byref(e), 1 if add_forces else 0), "ewald_exact")
    return e.value


def errorEstimatePME(sys, K, beta, rcut):
    """(err_dir, err_rec) of ElectrostaticInteraction::errorEstimatePME."""
    KK = (C.c_int * 3)(*[int(k) for k in K])
    d, r = C.c_double(), C.c_double()
    check(lib.md_error_estimate_pme(sys.h, KK, float(beta), float(rcut), C.byref(d), C.byref(r)), "errorEstimatePME")
    return d.value, r.value


def errorEstimateInterpolRec(sys, K, order, beta):
    """ik-SPME interpolation estimate of ElectrostaticInteraction_rec_BSpline::errorEstimate."""
    KK = (C.c_int * 3)(*[int(k) for k in K])
    e = C.c_double()
    check(lib.md_error_estimate_spme_ik(sys.h, KK, int(order), float(beta), C.byref(e)), "errorEstimate")
    return e.value


class ErrorEstimate_SPME_Ik:
    """ErrorEstimate_SPME_Ik (analyze tools): reinit(beta, order, dp) builds the
    kernel on the grid K of box L; calError(charge) gives error1 and error2
    ([K..., 2]); rms() the RMS force error per grid point."""

    def __init__(self, K, L, beta, order, device=0):
        h = C.c_void_p()
        KK = (C.c_int * 3)(*[int(k) for k in K])
        LL = (C.c_double * 3)(*[float(x) for x in L])
        check(lib.md_errmap_create(C.byref(h), KK, LL, float(beta), int(order), int(device)),
              "ErrorEstimate_SPME_Ik")
        self.h = h
        self.K = tuple(int(k) for k in K)

    def __del__(self):
        if getattr(self, "h", None):
            lib.md_errmap_destroy(self.h)
            self.h = None

    def set_profile(self, rho1, rho2):
        a = _f64(rho1).reshape(-1)
        b = _f64(rho2).reshape(-1)
        check(lib.md_errmap_set_profile(self.h, _p(a), _p(b)), "set_profile")

    def deposit(self, sys):
        check(lib.md_errmap_deposit(self.h, sys.h), "deposit")

    def profile(self):
        a = np.empty(self.K)
        b = np.empty(self.K)
        check(lib.md_errmap_get_profile(self.h, _p(a), _p(b)), "profile")
        return a, b

    def calError(self, charge=1.0):
        e1 = np.empty(self.K + (2,))
        e2 = np.empty(self.K + (2,))
        check(lib.md_errmap_compute(self.h, float(charge), _p(e1), _p(e2)), "calError")
        return e1, e2

    def rms(self, charge=1.0):
        e1, e2 = self.calError(charge)
        return np.sqrt(e1[..., 0] + e2[..., 0])

    def mean_force(self, charge=1.0):
        """The signed mean force error field e1_d (print_meanf): [3, K...]."""
        out = np.empty((3,) + self.K)
        check(lib.md_errmap_mean_force(self.h, float(charge), _p(out)), "mean_force")
        return out


class ErrorEstimate_dir(ErrorEstimate_SPME_Ik):
    """ErrorEstimate_dir (analyze tools): reinit(beta, rcut, dp) builds the
    real-space kernels on the grid K of box L; calError / rms as for the ik map."""

    def __init__(self, K, L, beta, rcut, device=0):
        h = C.c_void_p()
        KK = (C.c_int * 3)(*[int(k) for k in K])
        LL = (C.c_double * 3)(*[float(x) for x in L])
        check(lib.md_errmap_create_dir(C.byref(h), KK, LL, float(beta), float(rcut), int(device)),
              "ErrorEstimate_dir")
        self.h = h
        self.K = tuple(int(k) for k in K)


class ErrorEstimate_SPME_Ana(ErrorEstimate_SPME_Ik):
    """ErrorEstimate_SPME_Ana (analyze tools): reinit(beta, order, dp) builds the
    analytic-differentiation kernel on the grid K of box L; calError(charge)
    gives error1 and error2 ([K..., 2]); the RMS force error adds the self term
    self_error * charge^4."""

    def __init__(self, K, L, beta, order, device=0):
        h = C.c_void_p()
        KK = (C.c_int * 3)(*[int(k) for k in K])
        LL = (C.c_double * 3)(*[float(x) for x in L])
        check(lib.md_errmap_create_ana(C.byref(h), KK, LL, float(beta), int(order), int(device)),
              "ErrorEstimate_SPME_Ana")
        self.h = h
        self.K = tuple(int(k) for k in K)
        self.L = tuple(float(x) for x in L)

    def self_error(self):
        v = C.c_double()
        check(lib.md_errmap_self_error(self.h, C.byref(v)), "self_error")
        return v.value

    def qself_error(self, charge=1.0):
        return self.self_error() * charge ** 4

    def rms(self, charge=1.0):
        e1, e2 = self.calError(charge)
        return np.sqrt(e1[..., 0] + e2[..., 0] + self.qself_error(charge))

    def fconv(self, k):
        """FConvRho1_{x,y,z} for alias index k (0 < |k| <= 2): [3, K..., 2]."""
        out = np.empty((3,) + self.K + (2,))
        check(lib.md_errmap_ana_fconv(self.h, int(k), _p(out)), "fconv")
        return out

    def print_error(self, path, charge=1.0):
        """The columns of ErrorEstimate_SPME_Ana::print_error along x at y = z = 0:
        x, RMS, error1 (re, im), error2 (re, im), self error, and the k = 1
        x-kernel terms of FConvRho1 (taken, as the reference does, at the
        grid's linear index i)."""
        e1, e2 = self.calError(charge)
        q = self.qself_error(charge)
        fc = self.fconv(1)[0].reshape(-1, 2)
        Kx, Lx = self.K[0], self.L[0]
        c = 4.0 * np.pi ** 2 * Kx * Kx * (1.0 / Lx) ** 2
        with open(path, "w") as f:
            f.write("# 1      2         3-4       5-6      7\n")
            f.write("# x  RMS-E  E_inhomo^2  E_homo^2  selfE^2\n")
            for i in range(Kx):
                a, b = e1[i, 0, 0], e2[i, 0, 0]
                f.write("%f %e   %e %e %e %e   %e %e %e\n" % (
                    (i + 0.5) * Lx / Kx, np.sqrt(a[0] + b[0] + q), a[0], a[1], b[0], b[1], q,
                    np.sqrt(c * fc[i, 0] ** 2), np.sqrt(c * fc[i, 1] ** 2)))


class GroConf:
    """A .gro configuration (GromacsFileManager::readGroFile): residue and atom
    indices, names (str), positions and velocities [N, 3] and the box edges."""

    def __init__(self, pos, box, vel=None, resd_index=None, resd_name=None, atom_name=None,
                 atom_index=None, title=""):
        self.pos = _f64(pos).reshape(-1, 3)
        n = self.pos.shape[0]
        self.box = _f64(box, (3,))
        self.vel = np.zeros((n, 3)) if vel is None else _f64(vel).reshape(-1, 3)
        self.resd_index = np.arange(1, n + 1, dtype=np.int32) if resd_index is None else \
            np.ascontiguousarray(resd_index, np.int32)
        self.atom_index = np.arange(1, n + 1, dtype=np.int32) if atom_index is None else \
            np.ascontiguousarray(atom_index, np.int32)
        self.resd_name = [""] * n if resd_name is None else list(resd_name)
        self.atom_name = [""] * n if atom_name is None else list(atom_name)
        self.title = title

    @property
    def n(self):
        return self.pos.shape[0]


def _names_to_slots(names):
    out = np.zeros((len(names), 8), np.uint8)
    for i, s in enumerate(names):
        b = s.encode()[:7]
        out[i, :len(b)] = np.frombuffer(b, np.uint8)
    return out


def read_gro(path):
    """GromacsFileManager::readGroFile (values pass through binary32 as in the reference)."""
    n = C.c_int()
    check(lib.md_gro_count(str(path).encode(), C.byref(n)), "read_gro")
    n = n.value
    ri = np.zeros(n, np.int32)
    ai = np.zeros(n, np.int32)
    rn = np.zeros((n, 8), np.uint8)
    an = np.zeros((n, 8), np.uint8)
    pos = np.zeros((n, 3))
    vel = np.zeros((n, 3))
    box = np.zeros(3)
    check(lib.md_gro_read(str(path).encode(), n, _p(ri, C.c_int), _p(rn, C.c_char), _p(an, C.c_char),
                          _p(ai, C.c_int), _p(pos), _p(vel), _p(box)), "read_gro")
    with open(path, "rb") as f:
        title = f.readline().decode(errors="replace").rstrip("\n")
    dec = lambda row: bytes(row).split(b"\0", 1)[0].decode()
    return GroConf(pos, box, vel, ri, [dec(r) for r in rn], [dec(r) for r in an], ai, title)


def write_gro(path, conf, title=None):
    """GromacsFileManager::writeGroFile with the given first line."""
    rn = _names_to_slots(conf.resd_name)
    an = _names_to_slots(conf.atom_name)
    t = conf.title if title is None else title
    check(lib.md_gro_write(str(path).encode(), t.encode(), conf.n, _p(conf.resd_index, C.c_int),
                           _p(rn, C.c_char), _p(an, C.c_char), _p(conf.atom_index, C.c_int),
                           _p(_f64(conf.pos)), _p(_f64(conf.vel)), _p(_f64(conf.box))), "write_gro")


def system_from_gro(path, charge=None, mass=None, precision=PREC_MIXED, device=0):
    """MDSystem::initConfig(configfile) + initDeviceData: the system and the
    configuration it was read from (names and indices for writing it back)."""
    conf = read_gro(path)
    return MDSystem(conf.pos, conf.box, vel=conf.vel, charge=charge, mass=mass, precision=precision,
                    device=device), conf


def write_system_gro(path, sys, conf, step=0, time=0.0):
    """MDSystem::writeHostDataGro: the system's current positions (wrapped, original
    order), velocities and box with the names of conf, titled as the reference does."""
    out = GroConf(sys.positions(), sys.box(), sys.velocities(), conf.resd_index, conf.resd_name,
                  conf.atom_name, conf.atom_index)
    write_gro(path, out, "# at time = %f, step = %d" % (time, step))


def check_grid_barrier(sys, skip_block=-1, limit_s=1.0):
    """Runs the fused rebuild's grid barrier once (a block per SM) on the
    system's state; with skip_block >= 0 that block never arrives and the
    others give up after limit_s.  Returns True when the barrier timed out;
    the timeout flag is cleared again and the system stays usable."""
    t = C.c_int()
    check(lib.md_check_grid_barrier(sys.h, int(skip_block), float(limit_s), C.byref(t)), "check_grid_barrier")
    return bool(t.value)


def choose_beta(sys, rcut, target):
    b = C.c_double()
    check(lib.md_choose_beta(sys.h, float(rcut), float(target), C.byref(b)), "choose_beta")
    return b.value


def choose_spme_params(sys, rcut, order, target, kmax=1024):
    """(beta, K, err_dir, err_rec): splitting parameter and power-of-two mesh whose
    largest per-bin error estimates (real space at the densest region; ik-SPME map
    ErrorEstimate_SPME_Ik of the system's charge profile) are within target/sqrt(2)
    each (md_choose_spme_params)."""
    b, ed, er = C.c_double(), C.c_double(), C.c_double()
    K = (C.c_int * 3)()
    check(lib.md_choose_spme_params(sys.h, float(rcut), int(order), float(target), int(kmax), C.byref(b), K,
                                    C.byref(ed), C.byref(er)), "choose_spme_params")
    return b.value, tuple(K), ed.value, er.value


class AssignRCut:
    """Per-atom cutoff from an rc lattice (AssignRCut::getRCut + assign)."""

    def __init__(self, lattice):
        self.lattice = np.ascontiguousarray(lattice, dtype=np.float32)
        assert self.lattice.ndim == 3

    def uniform(self, sys, rc):
        check(lib.md_set_rcut_uniform(sys.h, float(rc)), "AssignRCut::uniform")

    def assign(self, sys):
        nx, ny, nz = self.lattice.shape
        check(lib.md_assign_rcut(sys.h, _p(self.lattice, C.c_float), nx, ny, nz), "AssignRCut::assign")


class VelocityVerlet:
    def __init__(self, sys):
        self.sys = sys

    def step1(self, sys, dt):
        check(lib.md_vv_step1(sys.h, float(dt)), "VelocityVerlet::step1")

    def step2(self, sys, dt, with_stats=True):
        check(lib.md_vv_step2(sys.h, float(dt), 1 if with_stats else 0), "VelocityVerlet::step2")


def langevin_params(dt, temperature, gamma_t, tau_p=0.0, kappa_t=0.0, p_ref=(0.0, 0.0, 0.0),
                    npt_dirs=0, seed=1):
    p = LangevinParams()
    p.dt, p.temperature, p.gamma_t, p.tau_p, p.kappa_t = dt, temperature, gamma_t, tau_p, kappa_t
    for d in range(3):
        p.p_ref[d] = p_ref[d]
    p.npt_dirs = npt_dirs
    p.seed = seed
    return p


class Langevin:
    """Langevin NVT / NPT (langevin.npt/writedown/paper.tex:355-369, 586-600)."""

    def __init__(self, sys, **kw):
        self.params = langevin_params(**kw)
        check(lib.md_langevin_setup(sys.h, C.byref(self.params)), "Langevin")
        self.sys = sys

    def step1(self, nlist=None):
        check(lib.md_langevin_step1(self.sys.h, nlist.h if nlist else None), "Langevin::step1")

    def step2(self):
        check(lib.md_langevin_step2(self.sys.h), "Langevin::step2")


class AdaptRCutEstimator:
    """AdaptRCut + DensityProfile_PiecewiseConst + PressureCorrection on the GPU
    (ENG/src/AdaptRCut.cu, ENG/src/DensityProfile.cu, ENG/src/PressureCorrection.cu)."""

    def __init__(self, sys, refh=1.0, rcmin=2.5, rcmax=5.0, rcstep=0.5):
        h = C.c_void_p()
        check(lib.md_arc_create(C.byref(h), sys.h, refh, rcmin, rcmax, rcstep), "AdaptRCut")
        self.h = h
        self.sys = sys
        n = (C.c_int * 3)()
        nrc = C.c_int()
        check(lib.md_arc_get_dims(h, n, C.byref(nrc)), "dims")
        self.n = tuple(n)
        self.nrc = nrc.value
        self.nele = self.n[0] * self.n[1] * self.n[2]
        self.rc_list = np.array([rcmin + i * rcstep for i in range(self.nrc)])

    def __del__(self):
        if getattr(self, "h", None):
            lib.md_arc_destroy(self.h)
            self.h = None

    def deposite(self, sys=None):
        check(lib.md_arc_deposit(self.h, (sys or self.sys).h), "deposite")

    def clearData(self):
        check(lib.md_arc_clear_profile(self.h), "clearData")

    def set_profile(self, rho):
        a = _f64(rho).reshape(self.n)
        check(lib.md_arc_set_profile(self.h, _p(a)), "set_profile")

    def profile(self):
        a = np.empty(self.n, np.float64)
        check(lib.md_arc_get_profile(self.h, _p(a)), "profile")
        return a

    def update(self, prec, nrefine=0):
        """calError + calRCut(prec) + refineRCut x nrefine + PressureCorrection."""
        check(lib.md_arc_update(self.h, float(prec), int(nrefine)), "AdaptRCut::update")

    def error(self):
        a = np.empty((self.nrc,) + self.n, np.float64)
        check(lib.md_arc_get_error(self.h, _p(a)), "error")
        return a

    def rcut(self):
        rc = np.empty(self.n, np.float64)
        idx = np.empty(self.n, np.int32)
        err = np.empty(self.n, np.float64)
        check(lib.md_arc_get_rcut(self.h, _p(rc), _p(idx, C.c_int), _p(err)), "rcut")
        return rc, idx, err

    def tables(self):
        s1 = np.empty((self.nrc,) + self.n)
        s2 = np.empty((3, self.nrc) + self.n)
        pc = np.empty((3, self.nrc) + self.n)
        check(lib.md_arc_get_tables(self.h, _p(s1), _p(s2), _p(pc)), "tables")
        return s1, s2, pc

    def assign(self, sys=None):
        check(lib.md_arc_assign(self.h, (sys or self.sys).h), "AssignRCut::assign")

    def pressure_correction(self, sys=None):
        out = np.zeros(3)
        check(lib.md_arc_pressure_correction(self.h, (sys or self.sys).h, _p(out)), "pressure_correction")
        return out


class ForceCorr:
    """Long-range LJ force correction (LFC) of the fcorr tools: ForceCorr
    (FCR/src/ForceCorr.cu) on a DensityProfile_PiecewiseConst(box, refh) and
    AssignForceCorr (FCR/src/AssignForceCorr.cu), on the GPU.  reinit(rc, dp) is
    the constructor; update() is dp.calculate + calError + getForceCorr; assign()
    gives every atom its bin's value, which the engine adds to the forces once
    set with InteractionEngine.setForceCorrection."""

    def __init__(self, sys, rc, refh=1.0):
        h = C.c_void_p()
        check(lib.md_fcorr_create(C.byref(h), sys.h, float(rc), float(refh)), "ForceCorr")
        self.h = h
        self.sys = sys
        self.rc = float(rc)
        n = (C.c_int * 3)()
        check(lib.md_fcorr_get_dims(h, n), "dims")
        self.n = tuple(n)
        self.nele = self.n[0] * self.n[1] * self.n[2]

    def __del__(self):
        if getattr(self, "h", None):
            lib.md_fcorr_destroy(self.h)
            self.h = None

    def deposite(self, sys=None):
        check(lib.md_fcorr_deposit(self.h, (sys or self.sys).h), "deposite")

    def clearData(self):
        check(lib.md_fcorr_clear_profile(self.h), "clearData")

    def set_profile(self, rho):
        a = _f64(rho).reshape(self.n)
        check(lib.md_fcorr_set_profile(self.h, _p(a)), "set_profile")

    def profile(self):
        a = np.empty(self.n, np.float64)
        check(lib.md_fcorr_get_profile(self.h, _p(a)), "profile")
        return a

    def update(self):
        check(lib.md_fcorr_update(self.h), "ForceCorr::calError")

    def zero(self):
        check(lib.md_fcorr_zero(self.h), "AssignForceCorr::zero")

    def field(self):
        """(re, im): error2r{x,y,z} on the bins, each (3, nx, ny, nz)"""
        re = np.empty((3,) + self.n)
        im = np.empty((3,) + self.n)
        check(lib.md_fcorr_get_field(self.h, _p(re), _p(im)), "field")
        return re, im

    def assign(self, sys=None):
        check(lib.md_fcorr_assign(self.h, (sys or self.sys).h), "AssignForceCorr::assign")

    def values(self):
        """per-atom correction [N][3], original atom order"""
        v = np.empty((self.sys.n, 3))
        check(lib.md_fcorr_get_values(self.h, _p(v)), "values")
        return v


class NoseHoover_Chains2:
    """NoseHoover_Chains2 (ENG/include/Thermostat.h:77-120): reinit(sys, refT, tauT),
    operator_L(dt, sys), HamiltonianContribution(); step1/step2 give the
    lj.nhc-xtc step (COM removal, operator_L(dt/2), VV step1 | forces | VV step2,
    operator_L(dt/2))."""

    def __init__(self, sys, ref_T, tau_T, remove_com=True):
        h = C.c_void_p()
        check(lib.md_nhc_create(C.byref(h), sys.h, float(ref_T), float(tau_T), 1 if remove_com else 0),
              "NoseHoover_Chains2")
        self.h = h
        self.sys = sys

    def __del__(self):
        if getattr(self, "h", None):
            lib.md_nhc_destroy(self.h)
            self.h = None

    def operator_L(self, dt, sys=None, with_stats=True):
        check(lib.md_nhc_operator_L(self.h, (sys or self.sys).h, float(dt), 1 if with_stats else 0), "operator_L")

    def step1(self, dt, nlist=None):
        check(lib.md_nhc_step1(self.h, self.sys.h, nlist.h if nlist is not None else None, float(dt)), "step1")

    def step2(self, dt):
        check(lib.md_nhc_step2(self.h, self.sys.h, float(dt)), "step2")

    def state(self):
        out = np.zeros(5)
        check(lib.md_nhc_get_state(self.h, _p(out)), "state")
        return out

    def HamiltonianContribution(self):
        return float(self.state()[4])


class NoseHoover_Chains2_Isobaric:
    """NoseHoover_Chains2_Isobaric (ENG/include/Barostat.h:90-175): reinit(sys, refT,
    tauT, refP, tauP, pressureCorr) and the operators L_CP, L_v, L_r, L_box."""

    def __init__(self, sys, ref_T, tau_T, ref_P, tau_P, pressure_corr=0.0):
        h = C.c_void_p()
        check(lib.md_nhc_npt_create(C.byref(h), sys.h, float(ref_T), float(tau_T), float(ref_P), float(tau_P),
                                    float(pressure_corr)), "NoseHoover_Chains2_Isobaric")
        self.h = h
        self.sys = sys

    def __del__(self):
        if getattr(self, "h", None):
            lib.md_nhc_npt_destroy(self.h)
            self.h = None

    def operator_L_CP(self, dt):
        check(lib.md_nhc_npt_operator_L_CP(self.h, self.sys.h, float(dt)), "operator_L_CP")

    def operator_L_v(self, dt):
        check(lib.md_nhc_npt_operator_L_v(self.h, self.sys.h, float(dt)), "operator_L_v")

    def operator_L_r(self, dt):
        check(lib.md_nhc_npt_operator_L_r(self.h, self.sys.h, float(dt)), "operator_L_r")

    def operator_L_box(self, dt):
        check(lib.md_nhc_npt_operator_L_box(self.h, self.sys.h, float(dt)), "operator_L_box")

    def state(self):
        out = np.zeros(5)
        check(lib.md_nhc_npt_get_state(self.h, _p(out)), "state")
        return out


class Simulation:
    """Graph-captured Langevin MD driver (the hot loop of ENG/app/lj.nhc-xtc.cu)."""

    def __init__(self, sys, engine, skin, cell_size, lv, nl_mode=NL_MINIMAGE, expansion=1.5,
                 use_graph=True, max_rcut=0.0, integrator="langevin", nhc_tau=0.0, remove_com=True,
                 spme=None):
        """integrator "langevin" (lv: BAOAB NVT/NPT) or "nhc" (the lj.nhc-xtc step:
        2-chain Nose-Hoover at lv.temperature with period nhc_tau, velocity Verlet with
        step lv.dt, COM velocity removed every step when remove_com).  spme: an SPME
        of the same system whose reciprocal forces are added every step (with the
        engine's real-space Ewald, registCoulomb, this is the full Ewald split)."""
        p = SimParams()
        p.lv = lv
        p.skin = skin
        p.cell_size = cell_size
        p.expansion = expansion
        p.nl_mode = nl_mode
        p.use_graph = 1 if use_graph else 0
        p.stats_every = 1
        p.max_rcut = max_rcut
        p.integrator = {"langevin": INTEG_LANGEVIN, "nhc": INTEG_NHC}[integrator]
        p.nhc_tau = nhc_tau
        p.remove_com = 1 if remove_com else 0
        p.spme = spme.h if spme is not None else None
        self._spme = spme  # keep the SPME alive as long as the driver
        self.params = p
        h = C.c_void_p()
        check(lib.md_sim_create(C.byref(h), sys.h, engine.h, C.byref(p)), "Simulation")
        self.h = h
        self.sys = sys
        self.engine = engine

    def __del__(self):
        if getattr(self, "h", None):
            lib.md_sim_destroy(self.h)
            self.h = None

    def run(self, nsteps):
        check(lib.md_sim_run(self.h, int(nsteps)), "Simulation::run")

    def set_stats_ring(self, rows):
        """Every step's statistic slots written by the device into rows
        (float64 [R, STAT_COUNT], page-locked for a copy without registration),
        row k mod R for the k-th step from now; None detaches."""
        if rows is None:
            check(lib.md_sim_set_stats_ring(self.h, None, 0), "set_stats_ring")
            self._ring = None
            return
        if rows.dtype != np.float64 or rows.ndim != 2 or rows.shape[1] != STAT_COUNT or not rows.flags.c_contiguous:
            raise ValueError("set_stats_ring: rows must be a contiguous float64 [R, STAT_COUNT] array")
        check(lib.md_sim_set_stats_ring(self.h, _p(rows), rows.shape[0]), "set_stats_ring")
        self._ring = rows

    def counters(self):
        s, r, f = C.c_int64(), C.c_int64(), C.c_int()
        check(lib.md_sim_counters(self.h, C.byref(s), C.byref(r), C.byref(f)), "counters")
        return s.value, r.value, f.value

    def uses_conditional_graph(self):
        v = C.c_int()
        check(lib.md_sim_uses_conditional_graph(self.h, C.byref(v)), "conditional")
        return bool(v.value)

    def rebuild_kind(self):
        """How a step decides on the device whether to rebuild the lists:
        "fused" (one cooperative kernel gated by the device's rebuild flag),
        "conditional" (the chain of kernels under a conditional graph node) or
        "gated" (the chain launched every step, each kernel gated)."""
        v = C.c_int()
        check(lib.md_sim_rebuild_kind(self.h, C.byref(v)), "rebuild kind")
        return {0: "gated", 1: "conditional", 2: "fused"}[v.value]

    def set_rebuild_kind(self, kind):
        """"fused" (the default where the device can run it) or "conditional"
        (the chain of kernels); both give the same lists bit for bit."""
        k = {"fused": 2, "conditional": 1}[kind]
        check(lib.md_sim_set_rebuild_kind(self.h, k), "set rebuild kind")

    def nhc_state(self):
        """xi1, xi2, vxi1, vxi2, HamiltonianContribution of the driver's chain."""
        out = np.zeros(5)
        check(lib.md_sim_get_nhc_state(self.h, _p(out)), "nhc_state")
        return out

    def attach_force_corr(self, fc, assign_every=40, sample_every=40, update_every=2000):
        """assignForceCorrFeq / densityProfileSamplingFeq / updateForceCorrFeq of the
        fcorr app (FCR/app/lj.nhc-xtc.cu:50-51, 172-227); sets it on the engine."""
        check(lib.md_sim_attach_force_corr(self.h, fc.h, int(assign_every), int(sample_every), int(update_every)),
              "attach_force_corr")
        self.fcorr = fc

    def attach_adapt_rcut(self, arc, sample_every=40, update_every=2000, prec=0.02, nrefine=0):
        """rcutAssignFeq / densityProfileSamplingFeq / rcutUpdateFeq of lj.nhc-xtc.cu."""
        check(lib.md_sim_attach_adapt_rcut(self.h, arc.h, sample_every, update_every, prec, nrefine),
              "attach_adapt_rcut")
        self.arc = arc
