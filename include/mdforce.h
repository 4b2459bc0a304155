/*
 * mdforce.h -- C ABI of the B200 (sm_100a) molecular-dynamics force path.
 *
 * This is the drop-in boundary for the interaction-engine API of the
 * md.error GPU engine (shortRange.inhomo/template/tools/simulation.*).
 * Every entry point is plain C: opaque handles, raw pointers and sizes,
 * no C++ or torch types.  Each call names the reference interface it
 * replaces.  Paths are relative to the md.error project root;
 * "ENG" = shortRange.inhomo/template/tools/simulation.hetero.cutoff,
 * "UNI" = shortRange.inhomo/template/tools/simulation.uniform.cutoff,
 * "RE"  = longRange.hetero/profile.test/template/tools/real.error.
 *
 * Conventions
 *  - Every function returns an int status (MD_OK == 0).  No exception
 *    crosses the ABI.  md_last_error_message() gives the detail of the
 *    last failure on the calling thread.
 *  - Host arrays of per-atom vectors are [N][3] row-major doubles in the
 *    ORIGINAL atom order given at md_system_create; the library keeps
 *    atoms in cell order on the device and un-permutes on the way out.
 *  - All device work of a system is issued on the system's stream
 *    (md_system_set_stream); calls return without synchronising unless
 *    they copy results to the host.
 *  - Handles are not thread-safe: one handle per host thread.
 */
#ifndef MDFORCE_H
#define MDFORCE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes: the first three mirror mdError_t (ENG/include/error.h:19-26) */
enum md_status {
  MD_OK = 0,
  MD_ERR_CELL_OVERFLOW = 1,   /* mdErrorShortCellList                        */
  MD_ERR_NLIST_OVERFLOW = 2,  /* mdErrorShortNeighborList                    */
  MD_ERR_CELL_INDEX = 3,      /* mdErrorOverFlowCellIdx                      */
  MD_ERR_CUDA = 10,           /* a CUDA runtime call failed (MDExcptCuda)     */
  MD_ERR_BADARG = 11,         /* invalid argument / NaN input                 */
  MD_ERR_UNSUPPORTED = 12,    /* feature absent (e.g. bonded terms present)   */
  MD_ERR_TIMEOUT = 13,        /* a bounded device wait gave up                */
  MD_ERR_NOMEM = 14,
  MD_ERR_IO = 15              /* a file could not be opened, read or written (MDExcptCannotOpenFile,
                                 MDExcptWrongFileFormat) */
};

/* arithmetic of the force path */
enum md_precision {
  MD_PREC_MIXED = 0, /* FP32 positions and pair math, FP64 / compensated accumulation */
  MD_PREC_FP64 = 1   /* plain FP64 everywhere                                         */
};

/* neighbour-list criterion (both are bit-exact restatements in binary32) */
enum md_nlist_mode {
  /* ENG buildDeviceNeighborList_AllPair (ENG/src/NeighborList.cu:327-420):
     d = r_j - r_i, d -= floorf(d/L + 0.5) L, keep if |d|^2 < (rcut_i + skin)^2 */
  MD_NL_MINIMAGE = 0,
  /* UNI buildDeviceNeighborList_DeviceCellList
     (UNI/src/NeighborList_interface.cu:361-491): d = (r_j - shift) - r_i with the
     periodic shift of j's cell, keep if |d|^2 < rlist^2 */
  MD_NL_CELLSHIFT = 1
};

/* statistic slots, FP64 (MDStatistic slots, ENG/include/Statistic.h) */
enum md_stat_slot {
  MD_STAT_NB_ENERGY = 0,   /* mdStatisticNonBondedPotential  */
  MD_STAT_VIRIAL_XX = 1,   /* mdStatisticVirialXX (sum f.d)  */
  MD_STAT_VIRIAL_YY = 2,
  MD_STAT_VIRIAL_ZZ = 3,   /* (virials include every force term of the step) */
  MD_STAT_ELEC_DIR = 4,    /* real-space Ewald energy        */
  MD_STAT_KINETIC_XX = 5,  /* 1/2 sum m v_x^2                */
  MD_STAT_KINETIC_YY = 6,
  MD_STAT_KINETIC_ZZ = 7,
  MD_STAT_PRESSURE_CORR_XX = 8, /* tail corrections added to P  */
  MD_STAT_PRESSURE_CORR_YY = 9,
  MD_STAT_PRESSURE_CORR_ZZ = 10,
  MD_STAT_ELEC_REC = 11,   /* reciprocal (SPME) energy       */
  MD_STAT_ELEC_SELF = 12,  /* -beta/sqrt(pi) sum q^2         */
  MD_STAT_BOND_ENERGY = 13, /* mdStatisticBondedPotential: bonds and angles */
  MD_STAT_COUNT = 16
};

typedef struct md_system md_system;
typedef struct md_cell_list md_cell_list;
typedef struct md_nlist md_nlist;
typedef struct md_engine md_engine;

/* Last error text of the calling thread (never NULL). */
const char* md_last_error_message(void);
/* Library version string. */
const char* md_version(void);
/* Number of CUDA devices visible (0 on a host without GPUs).  Makes no
   other CUDA call, so it is safe on CPU-only hosts. */
int md_device_count(int* out);

/* ------------------------------------------------------------------ system
 * Replaces MDSystem::initConfig / initDeviceData (ENG/include/MDSystem_interface.h:18-104,
 * ENG/include/MDSystem.h:43-78).  pos/vel are [N][3]; type, charge, mass are [N]
 * (vel, type, charge, mass may be NULL: zero velocity, type 0, charge 0, mass 1). */
int md_system_create(md_system** out, int n_atoms, const double box[3],
                     const double* pos, const double* vel, const int* type,
                     const double* charge, const double* mass, int precision,
                     int device);
int md_system_destroy(md_system* sys);
/* cudaStream_t passed as void*; NULL = the library's own stream (to use the
   legacy default stream, e.g. torch's default stream, pass cudaStreamLegacy). */
int md_system_set_stream(md_system* sys, void* cuda_stream);
int md_system_synchronize(md_system* sys);
int md_system_num_atoms(const md_system* sys, int* out);
int md_system_set_positions(md_system* sys, const double* pos);
int md_system_get_positions(md_system* sys, double* pos);
/* unwrapped positions: pos + image * L (MDSystem::recoverDeviceData) */
int md_system_get_unwrapped_positions(md_system* sys, double* pos);
int md_system_set_velocities(md_system* sys, const double* vel);
int md_system_get_velocities(md_system* sys, double* vel);
int md_system_get_forces(md_system* sys, double* force);
/* per-atom charges [N] in original order (MDSystem ddata.charge) */
int md_system_set_charges(md_system* sys, const double* charge);
/* Zero-copy input from device memory (e.g. torch tensors): raw device pointers in the
   caller's atom order; NULL members leave that quantity unchanged.  Asynchronous on the
   system's stream, which must be the producer's stream (md_system_set_stream) or ordered
   after it.  (The md_device_view of the survey's drop-in boundary: a DeviceMDData view.) */
typedef struct md_device_view {
  const double* pos;     /* [N][3] positions */
  const double* charge;  /* [N] charges */
} md_device_view;
int md_system_set_device_view(md_system* sys, const md_device_view* v);
int md_system_get_charges(md_system* sys, double* charge);
/* per-atom masses [N] in original order (MDSystem hdata.mass / massi, copied by
   MDSystem::initTopology, shortRange.inhomo/template/tools.collision/cal.real.error/src/
   MDSystem_interface.cu:125-127); every mass must be positive */
int md_system_set_masses(md_system* sys, const double* mass);
int md_system_get_masses(md_system* sys, double* mass);
int md_system_get_box(md_system* sys, double box[3]);
int md_system_set_box(md_system* sys, const double box[3]);
/* per-atom cutoff rcut_i in original order (MDSystem ddata.rcut) */
int md_system_set_rcut(md_system* sys, const float* rcut);
int md_system_get_rcut(md_system* sys, float* rcut);
/* Wrap every atom into [0,L) and update its image counters
   (normalizeSystem, ENG/src/BoxGeometry.cu:6-50). */
int md_system_normalize(md_system* sys);
/* atom types [N] in original order, 0 <= type < 16 (MDSystem hdata.type); 0 unless given */
int md_system_set_types(md_system* sys, const int* type);
int md_system_get_types(md_system* sys, int* type);
/* FP64 statistic slots (MDStatistic::updateHost); out has MD_STAT_COUNT entries. */
int md_system_read_stats(md_system* sys, double* out);
/* The same slots copied to out in stream order without waiting (out should be
   page-locked); out is valid after md_system_synchronize.  A per-step read of
   the statistics that does not stall the launch queue. */
int md_system_read_stats_async(md_system* sys, double* out);
int md_system_clear_stats(md_system* sys);

/* ------------------------------------------------------- configuration files
 * .gro files as the reference engine reads and writes them (GromacsFileManager::readGroFile /
 * writeGroFile, ENG/src/GromacsFileManager.cpp:7-124; MDSystem::initConfig and
 * writeHostDataGro, ENG/src/MDSystem_interface.cu:39-215).  Names are 8-byte slots
 * ([N][8], NUL padded; StringSize of the reference); pos / vel are [N][3].  Values pass
 * through binary32 both ways (the reference's ScalorType), so reading gives the reference's
 * values and writing gives its bytes.  An atom line without a velocity reads as zero
 * velocity.  Any of resd_index, resd_name, atom_name, atom_index, vel may be NULL (on
 * writing: indices 1..N, empty names, zero velocity).  File errors return MD_ERR_IO. */
int md_gro_count(const char* path, int* n_atoms);
int md_gro_read(const char* path, int n_atoms, int* resd_index, char* resd_name, char* atom_name,
                int* atom_index, double* pos, double* vel, double box[3]);
/* title is the first line without its newline (writeHostDataGro writes
   "# at time = %f, step = %d"); NULL writes an empty title */
int md_gro_write(const char* path, const char* title, int n_atoms, const int* resd_index,
                 const char* resd_name, const char* atom_name, const int* atom_index, const double* pos,
                 const double* vel, const double box[3]);

/* ------------------------------------------------------------- cell list
 * Replaces CellList(sys, cellSize, NThreadCell, NThreadAtom, bdir, divide) and
 * CellList::rebuild (ENG/include/CellList_interface.h:18-73,
 * UNI/src/CellList_interface.cu:147-251).  ncell_d = floor(L_d / cell_size) * divide
 * along the directions set in bdir (1=x,2=y,4=z), 1 elsewhere.  Rebuild bins every
 * atom (warp-aggregated atomics), then sorts all per-atom arrays into cell order
 * (counting sort, stable in the previous order) -- the Reshuffle step
 * (ENG/src/Reshuffle_interface.cu:40-102) is part of the rebuild. */
int md_cell_list_create(md_cell_list** out, md_system* sys, double cell_size,
                        int bdir, int divide);
int md_cell_list_destroy(md_cell_list* cl);
int md_cell_list_rebuild(md_cell_list* cl, md_system* sys);
int md_cell_list_get_ncell(md_cell_list* cl, int ncell[3]);
/* cell index (iz + ncz*(iy + ncy*ix), NeighborList.h D3toD1) of every atom,
   original order */
int md_cell_list_get_cell_index(md_cell_list* cl, md_system* sys, uint32_t* cell);

/* ------------------------------------------------------------ neighbour list
 * Replaces NeighborList(sysNbInter, sys, rlist, rlistExten, NThread, expansion) and
 * NeighborList::rebuild (ENG/include/NeighborList_interface.h:20-82).
 * mode MD_NL_MINIMAGE uses radius rcut_i + skin per atom; MD_NL_CELLSHIFT uses rlist.
 * capacity per atom = max(30, expansion * 4/3 pi rlist^3 rho) like
 * NeighborList::mallocDeviceNeighborList, raised by md_nlist_fit. */
int md_nlist_create(md_nlist** out, md_system* sys, double rlist, double skin,
                    double expansion, int mode);
int md_nlist_destroy(md_nlist* nl);
/* Builds from the cell list as last rebuilt: call md_cell_list_rebuild after the
   positions change and before this (as the reference app rebuilds clist before
   nlist); the build also uses each cell's z order taken at that rebuild. */
int md_nlist_rebuild(md_nlist* nl, md_system* sys, md_cell_list* cl);
/* Rebuild, and if any list overflowed grow the capacity to fit and rebuild
   again (host resize-and-retry of MD_ERR_NLIST_OVERFLOW). */
int md_nlist_fit(md_nlist* nl, md_system* sys, md_cell_list* cl);
int md_nlist_capacity(md_nlist* nl, int* out);
/* Displacement_max::calMaxDisplacemant (ENG/src/Displacement_interface.cu:80-126):
   max_i |r_i - r_i(last build)| (min image), FP64 on return. */
int md_nlist_max_displacement(md_nlist* nl, md_system* sys, double* out);
/* Total number of list entries (NeighborList::calSumNeighbor). */
int md_nlist_sum_neighbor(md_nlist* nl, md_system* sys, int64_t* out);
/* Export the lists in ORIGINAL indices: counts[N]; pairs receives, for every atom i
   in original order, its neighbours (original indices) back to back; pairs must
   hold the sum of counts (md_nlist_sum_neighbor). */
int md_nlist_get(md_nlist* nl, md_system* sys, int32_t* counts, int32_t* pairs);

/* ------------------------------------------------------- interaction engine
 * Replaces InteractionEngine(sys, NThread) / registNonBondedInteraction /
 * clearInteraction / applyNonBondedInteraction (ENG/include/InteractionEngine_interface.h:17-155,
 * ENG/src/InteractionEngine_interface.cu:317-380, 980-992, 1204-1281).
 * LJ 6-12 (LennardJones6_12, ENG/include/NonBondedInteraction.h:780-893):
 *   F_i = sum_j [|d|^2 < rcut_i^2] 4 eps (6 s^6/r^6 - 12 s^12/r^12)/r^2 d,  d = r_j - r_i
 *   E   = 1/2 sum_i sum_j [..] (4 eps (s^12/r^12 - s^6/r^6) + shift)
 * The cutoff is the per-atom rcut_i of the REFERENCE atom i only (asymmetric by design). */
int md_engine_create(md_engine** out, md_system* sys);
int md_engine_destroy(md_engine* eng);
int md_engine_register_lj(md_engine* eng, double epsilon, double sigma, double shift);
/* Several atom types (SystemNonBondedInteraction::add(t0, t1, LennardJones6_12Parameter)
 * with AtomNBForceTable::calForceIndex, ENG/include/NonBondedInteraction.h:673-683, and the
 * nbForce dispatch of ENG/include/NonBondedInteraction.h:469-495): LJ parameters for the
 * unordered pair (t0, t1), 0 <= t < 16.  Once a pair is given the non-bonded kernels look up
 * every pair's parameters by the two atoms' types, and pairs never given take no force and
 * no energy (mdForceNULL); md_engine_register_lj is then ignored.  The cutoff stays the
 * per-atom rcut_i.  Atom types come from md_system_create or md_system_set_types. */
int md_engine_register_lj_pair(md_engine* eng, int t0, int t1, double epsilon, double sigma, double shift);
/* The pair kinds of the nbForce dispatch, for a type pair; param[6] as the reference's
   *Parameter classes take them, unused entries 0 (the values of md_nb_kind are InteractionType's):
     MD_NB_LJ6_12       (eps, sigma, shift)             LennardJones6_12
     MD_NB_LJ6_12B      (eps, sigma, shift, rcut)       LennardJones6_12B: E = eps (s^12 - 2 s^6 + shift),
                                                        0 beyond rcut
     MD_NB_LJ6_12_CAP   (eps, sigma, shift, rcut, cap)  LennardJones6_12 with the force magnitude held at
                                                        cap inside the radius where it reaches cap
     MD_NB_LJ6_12B_CAP  (eps, sigma, shift, rcut, cap)  the same for the B form
     MD_NB_COSTAIL      (eps, b, wc)                    CosTail: WCA core of size b, -eps cos^2 tail of width wc
     MD_NB_COSTAIL_CAP  (eps, b, wc, cap)               CosTail with the capped core
     MD_NB_NULL         no interaction
   The cap radius is found as the reference finds it (0.95 steps, then bisection to 1e-4).
   A coincident pair (r = 0) takes no force from the capped kinds (the reference gives
   (-cap, 0, 0) there). */
enum md_nb_kind { MD_NB_NULL = 0, MD_NB_LJ6_12 = 1, MD_NB_LJ6_12_CAP = 2, MD_NB_COSTAIL = 3,
                  MD_NB_COSTAIL_CAP = 4, MD_NB_LJ6_12B = 5, MD_NB_LJ6_12B_CAP = 6 };
int md_engine_register_nb_pair(md_engine* eng, int t0, int t1, int kind, const double* param);
/* Bonded terms (SystemBondedInteraction::reinit + BondedInteractionList,
 * ENG/src/SystemBondedInteraction.cu:100-230; force functions ENG/include/BondInteraction.h:217-372,
 * ENG/include/AngleInteraction.h:365-1216; kernels calBondInteraction / calAngleInteraction,
 * ENG/src/InteractionEngine_interface.cu:1399-1775).  Atom indices are the original
 * (md_system_create) order.  Parameters are [n][3] as the *Parameter classes take them:
 *   MD_BOND_HARMONIC (k, r0):      F = k (1 - r0/r) d,     E = k/2 (r - r0)^2
 *   MD_BOND_FENE (k, rinf):        F = k rinf^2/(rinf^2 - r^2) d,  E = -k/2 rinf^2 ln(1 - r^2/rinf^2)
 *   MD_BOND_FENE2 (k, rs, r0):     the FENE form in r - r0 with range rs
 *   MD_ANGLE_HARMONIC (k, theta0): E = k (theta - theta0)^2 (atoms edge0, centre, edge1)
 *   MD_ANGLE_COS0 (k):             E = k (1 - cos(pi - theta))
 * with d = r_partner - r_self under the minimum image.  Each atom gathers its own
 * terms; the bonded energy goes to MD_STAT_BOND_ENERGY and the virial is added to the
 * non-bonded one.  A later call replaces the earlier set of that kind. */
enum md_bonded_type {
  MD_BOND_HARMONIC = 10000,   /* mdForceHarmonicSpring */
  MD_BOND_FENE = 10001,       /* mdForceFENE           */
  MD_BOND_FENE2 = 10002,      /* mdForceFENE2          */
  MD_ANGLE_HARMONIC = 20000,  /* mdForceAngleHarmonic  */
  MD_ANGLE_COS0 = 20001       /* mdForceCosAngle0      */
};
int md_engine_set_bonds(md_engine* eng, int n, const int* atoms /* [n][2] */, const int* type,
                        const double* param /* [n][3] */);
int md_engine_set_angles(md_engine* eng, int n, const int* atoms /* [n][3] edge0, centre, edge1 */,
                         const int* type, const double* param /* [n][3] */);
/* Exclusions (ExclusionList, ENG/include/ExclusionList.h): excluded pairs take no
   non-bonded force.  They are removed from the neighbour list after each build. */
int md_engine_set_exclusions(md_engine* eng, int n, const int* pairs /* [n][2] */);
/* the exclusion pass alone, for a list built before the exclusions were given */
int md_nlist_apply_exclusions(md_nlist* nl, md_system* sys);
/* registBondedInteraction: checks that n_bonds bonds were given to md_engine_set_bonds. */
int md_engine_register_bonded(md_engine* eng, int n_bonds);
int md_engine_clear_forces(md_engine* eng, md_system* sys);
/* with_stats 1 accumulates energy and diagonal virial into the FP64 slots;
   with_stats 2 runs the force kernel as the step driver does, leaving its
   statistics as per-warp rows that md_engine_finish_nonbonded_stats adds into
   the slots (the driver's closing kick adds them itself). */
int md_engine_apply_nonbonded(md_engine* eng, md_system* sys, md_nlist* nl, int with_stats);
int md_engine_finish_nonbonded_stats(md_engine* eng, md_system* sys);
/* applyBondedInteraction with statistics: adds the bonded forces to the system's forces
   (after md_engine_apply_nonbonded), stores MD_STAT_BOND_ENERGY and adds the virial;
   nothing to do without bonds or angles. */
int md_engine_apply_bonded(md_engine* eng, md_system* sys);
/* Real-space Ewald (ElectrostaticInteraction_dir, RE/src/EleDir.cpp:43-61) fused into
   the non-bonded kernel: E = 1/2 sum q_i q_j erfc(beta r)/r over the same list and
   cutoff; energy into MD_STAT_ELEC_DIR. */
int md_engine_register_coulomb(md_engine* eng, double beta);

/* ------------------------------------------------------------ long range
 * Reciprocal SPME, replaces ElectrostaticInteraction_rec_BSpline (ik differentiation,
 * RE/src/EleRecBSpline.cpp:393-877) and ElectrostaticInteraction_rec_FBSpline
 * (analytic differentiation, RE/src/EleRecFBSpline.cpp:771-1195): cardinal B-spline
 * order `order`, mesh K (powers of two), splitting beta, rectangular box.
 * method 0 = ik, 1 = analytic.  md_spme_apply adds the reciprocal forces and, with
 * stats, stores the energy in MD_STAT_ELEC_REC and adds its virial. */
typedef struct md_spme md_spme;
int md_spme_create(md_spme** out, md_system* sys, const int K[3], int order, double beta, int method);
int md_spme_destroy(md_spme* spme);
int md_spme_apply(md_spme* spme, md_system* sys, int with_stats);
/* the charge mesh Q (calQ) of the system's current positions, [K0][K1][K2] (spread on
 * demand; the force chain consumes its mesh in the first transform pass) */
int md_spme_get_mesh(md_spme* spme, double* Q);
/* Adjoint of the reciprocal SPME energy E = 1/2 sum_m psi(m) |Q^(m)|^2 (the energy of
 * ElectrostaticInteraction_rec_BSpline, RE/src/EleRecBSpline.cpp:393-536; no gradient
 * counterpart in the reference).  Recomputes spread and forward transform, then one
 * inverse transform of psi Q^ = Phi and a gather:
 *   dE_dq[i]      = sum_k theta_i(k) Phi(k)                    (electrostatic potential)
 *   dE_dr[i][d]   = q_i sum_k d theta_i(k)/du_d Phi(k) K_d/L_d  (exact gradient, = -F of
 *                   analytic differentiation whatever the force method)
 *   dE_dbeta      = sum_m 1/2 |Q^|^2 psi 2 pi^2 |m|^2 / beta^3
 *   dE_dpsi[t]    = 1/2 |Q^|^2 on the half spectrum [K0][K1][K2/2+1], the interior z
 *                   planes weighted 2 (each stands for m and -m), 0 at m = 0.
 * Every output is nullable; host arrays in original atom order; synchronises. */
int md_spme_energy_grad(md_spme* spme, md_system* sys, double* energy, double* dE_dq,
                        double* dE_dr, double* dE_dbeta, double* dE_dpsi);
/* md_spme_energy_grad with DEVICE outputs (energy, dE_dbeta: one double each; dE_dq [N],
   dE_dr [N][3] in the caller's atom order; each nullable), asynchronous on the system's
   stream: with md_system_set_device_view a differentiable SPME energy without host copies */
int md_spme_energy_grad_device(md_spme* spme, md_system* sys, double* energy, double* dE_dq, double* dE_dr,
                               double* dE_dbeta);
/* influence function psi on the half spectrum [K0][K1][K2/2+1] (calPsiFPhiF, ik scaling) */
int md_spme_get_influence(md_spme* spme, double* psi);
/* Self-force correction of analytic differentiation (SelfCorr::reinit + correction,
 * RE/src/SelfCorr.cpp:99-220, applied by RE/app/spme.cpp:266-270 for fbspline):
 * F_id -= sum_{k=1..3} c_d(k) q_i^2 sin(2 pi k K_d x_id / L_d), the c_d(k) from the
 * aliasing sums of the B-spline of the spme's order; added to the system's forces. */
int md_spme_self_correction(md_spme* spme, md_system* sys);
/* -beta/sqrt(pi) sum q^2 (ElectrostaticInteraction.cpp:219-222) into MD_STAT_ELEC_SELF */
int md_ewald_self_energy(md_system* sys, double beta, double* out);
/* Exact reciprocal Ewald sum over |m_d| <= K_d/2 in FP64 (ElectrostaticInteraction_rec_ES,
   RE/src/EleRecES.cpp:49-144): energy, and the forces added when add_forces != 0. */
int md_ewald_exact(md_system* sys, const int K[3], double beta, double* energy, int add_forces);

/* ------------------------------------------------------------ error estimates
 * ElectrostaticInteraction::errorEstimatePME (RE/src/ElectrostaticInteraction.cpp:349-401):
 * real-space and Ewald-truncation estimates with c2 = sum q^2 of the system; FP64 sums
 * on the device. */
int md_error_estimate_pme(md_system* sys, const int K[3], double beta, double rcut, double* err_dir,
                          double* err_rec);
/* ElectrostaticInteraction_rec_BSpline::errorEstimate (RE/src/EleRecBSpline.cpp:154-206):
 * homogeneous ik-SPME interpolation error for B-spline order `order`. */
int md_error_estimate_spme_ik(md_system* sys, const int K[3], int order, double beta, double* err);
/* Same estimate as md_error_estimate_spme_ik without allocating device memory, for
 * callers that reserve all device memory in their own pool or must keep the stream
 * allocator from growing between steps. No counterpart in the reference. Its scratch
 * is one fixed 180 KiB array per device: meshes up to K0*K1*K2 = 4,194,304 points
 * (larger ones give MD_ERR_BADARG). Each call looks the array's device address up,
 * waits for the system's stream and copies its tables from pageable host memory, so
 * it must not be called while that stream is being captured. Calls that overlap in
 * time on one device race on the shared scratch. */
int md_error_estimate_spme_ik_noalloc(md_system* sys, const int K[3], int order, double beta, double* err);
/* splitting beta whose real-space estimate equals target at cutoff rcut */
int md_choose_beta(md_system* sys, double rcut, double target, double* beta);
/* Splitting beta and power-of-two mesh K (at most kmax per axis) for an inhomogeneous
 * system so that the largest per-bin RMS force error estimate is within target / sqrt(2)
 * in real space and in reciprocal space (ik, B-spline order `order`).  No counterpart
 * function in the reference: it drives the reference's estimates the way their users pick
 * the parameters.  beta: errorEstimatePME's real-space term
 * (RE/src/ElectrostaticInteraction.cpp:349-401) at the largest local sum of q^2 per volume
 * over cubes of edge ~2 rcut.  K: grown from the homogeneous estimate
 * (RE/src/EleRecBSpline.cpp:154-206), then decided by the inhomogeneous ik-SPME map
 * (ErrorEstimate_SPME_Ik, as md_errmap_create) of the system's current charge profile on
 * each candidate mesh, coarsest axis doubled until within budget, finest axis halved
 * while within budget.  err_dir, err_rec (nullable): the two largest per-bin estimates.
 * Meshes stay within kmax per axis and 2^27 points; MD_ERR_BADARG when none meets the budget. */
int md_choose_spme_params(md_system* sys, double rcut, int order, double target, int kmax, double* beta,
                          int K[3], double* err_dir, double* err_rec);

/* Inhomogeneous ik-SPME error map (ErrorEstimate_SPME_Ik::reinit / calError,
 * longRange.hetero/profile.test/template/tools/analyze/src/ErrorEstimate_SPME_Ik.cpp:80-470,
 * as driven by analyze/app/error.spme.ik.cpp): on the grid K (the SPME mesh, also the
 * density-profile bins) of a rectangular box L, for B-spline order `order` and splitting
 * beta.  The kernel is built at creation (FP64 3D transforms on the device).  Profiles:
 * rho1 = density of charge signs (+1 / -1 per charge), rho2 = number density of charges,
 * [K0][K1][K2]; set explicitly or averaged over deposited samples of a system. */
typedef struct md_errmap md_errmap;
int md_errmap_create(md_errmap** out, const int K[3], const double L[3], double beta, int order,
                     int device);
int md_errmap_destroy(md_errmap* h);
int md_errmap_set_profile(md_errmap* h, const double* rho1, const double* rho2);
int md_errmap_deposit(md_errmap* h, md_system* sys);
int md_errmap_get_profile(md_errmap* h, double* rho1, double* rho2);
/* error1, error2 [K0][K1][K2][2] (real, imaginary) for charge magnitude `charge`; the
   RMS force error at a grid point is sqrt(error1[..][0] + error2[..][0]) (print_error) */
int md_errmap_compute(md_errmap* h, double charge, double* error1, double* error2);
/* Real-space map of the same form (ErrorEstimate_dir::reinit / calError,
 * analyze/src/ErrorEstimate_dir.cpp:70-331, driven by analyze/app/error.dir.cpp): kernels
 * s2k (vector) and s1k (scalar) of the erfc force beyond rcut, from the analyze tools'
 * adaptive Gauss-4 quadrature (tolerance 1e-20).  The quadrature needs erfc(beta rcut)
 * small; when it does not converge the call fails with MD_ERR_BADARG.  The handle takes
 * md_errmap_set_profile / deposit / compute like the ik map. */
int md_errmap_create_dir(md_errmap** out, const int K[3], const double L[3], double beta, double rcut,
                         int device);
/* Analytic-differentiation SPME map (ErrorEstimate_SPME_Ana::reinit / calKernel / calError,
 * analyze/src/ErrorEstimate_SPME_Ana.cpp:140-745, driven by analyze/app/error.spme.ana.cpp):
 * alias images 0 < |k| <= 2, the derivative-of-B-spline term in the second moment and a
 * homogeneous self-force error.  Takes md_errmap_set_profile / deposit / compute like the
 * ik map; the RMS force error at a grid point is
 * sqrt(error1[..][0] + error2[..][0] + self_error * charge^4) (print_error). */
int md_errmap_create_ana(md_errmap** out, const int K[3], const double L[3], double beta, int order,
                         int device);
/* self_error of the analytic map (0 for the other maps); multiply by charge^4 */
int md_errmap_self_error(md_errmap* h, double* out);
/* FConvRho1_{x,y,z} of the analytic map for alias index k (0 < |k| <= 2) and the current
   profile: IFFT(FFT(rho1 V/N) V F_d(k)) / V, out [3][K0][K1][K2][2] (print_error columns) */
int md_errmap_ana_fconv(md_errmap* h, int k, double* out);
/* print_meanf of the maps: the signed mean force error field
   e1_d = Re IFFT(k1_d FFT(rho1 V/N)) charge / V of the current profile, out [3][K0][K1][K2] */
int md_errmap_mean_force(md_errmap* h, double charge, double* out);

/* ------------------------------------------------------- per-atom cutoff
 * Replaces AssignRCut::getRCut + assign (ENG/src/AssignRCut.cu:46-117):
 * rcut_i = lattice[iz + nz*(iy + ny*ix)], ix = int((x*nx)/Lx) etc. (binary32). */
int md_assign_rcut(md_system* sys, const float* lattice, int nx, int ny, int nz);
int md_set_rcut_uniform(md_system* sys, float rc);

/* ------------------------------------------------------------ integrators
 * Velocity Verlet (ENG/src/Integrator.cu:273-436, VelocityVerlet::step1/step2). */
int md_vv_step1(md_system* sys, double dt);
int md_vv_step2(md_system* sys, double dt, int with_stats);

/* Langevin NVT / NPT from langevin.npt/writedown/paper.tex:355-369 (isotropic EOM)
   and :586-600 (anisotropic box), integrated by a BAOAB splitting with a
   counter-based Philox-4x32-10 normal stream keyed by (seed, step, atom id).
   npt_dirs: bit mask of box directions whose length fluctuates (4 = z only, the
   slab case with Pzz target); 0 = NVT.  gamma_t = 1/tau_T; M_h and gamma_P follow
   paper.tex:382-440: M = (tau_P/2pi)^2 A^2 / (kappa_T V0), gamma_P = 1/tau_P. */
typedef struct md_langevin_params {
  double dt, temperature, gamma_t;
  double tau_p, kappa_t, p_ref[3];
  int npt_dirs;
  uint64_t seed;
} md_langevin_params;
int md_langevin_setup(md_system* sys, const md_langevin_params* p);
/* first half of a step: B(dt/2) A(dt/2) O(dt) A(dt/2); also flags a rebuild when
   the displacement since the last list build exceeds skin/2 */
int md_langevin_step1(md_system* sys, md_nlist* nl);
/* second half: B(dt/2), kinetic tensor, barostat momentum half kick */
int md_langevin_step2(md_system* sys);
/* barostat state: box length velocity and momentum for each direction */
int md_langevin_get_state(md_system* sys, double* step, double p_h[3]);

/* Nose-Hoover chain of 2 thermostats (NoseHoover_Chains2, ENG/include/Thermostat.h:77-120,
 * ENG/src/Thermostat.cu:23-304): Q1 = tau_T^2 T 3N/(4 pi^2), Q2 = Q1/(3N), xi = 1, v_xi = 0
 * at creation; chain arithmetic in FP64 on the device.  remove_com: subtract the
 * centre-of-mass velocity at the start of every step (TranslationalFreedomRemover). */
typedef struct md_nhc md_nhc;
int md_nhc_create(md_nhc** out, md_system* sys, double ref_T, double tau_T, int remove_com);
int md_nhc_destroy(md_nhc* nhc);
/* NoseHoover_Chains2::operator_L(dt) on the current velocities; the kinetic tensor of the
   scaled velocities goes to MD_STAT_KINETIC_* */
int md_nhc_operator_L(md_nhc* nhc, md_system* sys, double dt, int with_stats);
/* manual stepping of the lj.nhc-xtc step: step1 = [COM removal] operator_L(dt/2) + VV step1
   + displacement test (nl nullable); step2 = VV step2 + operator_L(dt/2) */
int md_nhc_step1(md_nhc* nhc, md_system* sys, md_nlist* nl, double dt);
int md_nhc_step2(md_nhc* nhc, md_system* sys, double dt);
/* xi1, xi2, v_xi1, v_xi2 and HamiltonianContribution
   (Q1 v_xi1^2/2 + Q2 v_xi2^2/2 + 3N T xi1 + T xi2) */
int md_nhc_get_state(md_nhc* nhc, double out[5]);

/* Isobaric Nose-Hoover chain, isotropic box (NoseHoover_Chains2_Isobaric,
 * ENG/include/Barostat.h:90-175, ENG/src/Barostat.cu:6-460): Nf = 3N - 3,
 * Q1 = tau_T^2 T Nf, W = tau_P^2 T Nf, ep = ln(V)/3, vep = 0, xi1 = 1, vxi1 = 0.
 * The operators are the reference's; the pressure is tr(2/V (K - W_vir/2))/3 +
 * pressure_corr, from the current kinetic tensor and the virial slots of the last force
 * evaluation.  The reference composes no step from them; the standard MTK step is
 * L_CP(dt/2) L_v(dt/2) L_r(dt) L_box(dt) | forces | L_v(dt/2) L_CP(dt/2). */
typedef struct md_nhc_npt md_nhc_npt;
int md_nhc_npt_create(md_nhc_npt** out, md_system* sys, double ref_T, double tau_T, double ref_P,
                      double tau_P, double pressure_corr);
int md_nhc_npt_destroy(md_nhc_npt* h);
/* thermostat + barostat propagator L_CP(dt); kinetic tensor after scaling to the stats */
int md_nhc_npt_operator_L_CP(md_nhc_npt* h, md_system* sys, double dt);
/* v += dt F/m, kinetic tensor to the stats */
int md_nhc_npt_operator_L_v(md_nhc_npt* h, md_system* sys, double dt);
/* x = e^{vep dt} x + dt e^{vep dt/2} sinh-series(vep dt/2) v */
int md_nhc_npt_operator_L_r(md_nhc_npt* h, md_system* sys, double dt);
/* box edges *= e^{vep dt}, ep += vep dt */
int md_nhc_npt_operator_L_box(md_nhc_npt* h, md_system* sys, double dt);
/* ep, vep, xi1, vxi1, HamiltonianContribution (W vep^2/2 + Q1 vxi1^2/2 + (Nf+1) T xi1 + P V) */
int md_nhc_npt_get_state(md_nhc_npt* h, double out[5]);

/* ------------------------------------------------------------ simulation driver
 * Replaces the hot loop of ENG/app/lj.nhc-xtc.cu:159-274 for the Langevin path:
 * per step  [B A O A] -> (device-side rebuild check -> cell sort + list build) ->
 * clear -> LJ (+stats) -> [B] -> barostat.  The step is captured once into a CUDA
 * graph; the rebuild runs only when the device flag says so. */
typedef struct md_sim md_sim;
typedef struct md_sim_params {
  md_langevin_params lv;
  double skin;          /* Verlet skin (nlistExten)                       */
  double cell_size;     /* target cell edge (>= smallest list radius)      */
  double expansion;     /* list capacity factor                           */
  int nl_mode;          /* md_nlist_mode                                   */
  int use_graph;        /* capture the step in a CUDA graph                */
  int stats_every;      /* energy/virial every n steps (NPT needs 1)       */
  double max_rcut;      /* largest cutoff the run may assign (list capacity); 0 = current max */
  int integrator;       /* md_integrator: Langevin (lv) or Nose-Hoover chain + velocity Verlet */
  double nhc_tau;       /* NHC period tau_T (lv.temperature is the target, lv.dt the step) */
  int remove_com;       /* NHC: remove the centre-of-mass velocity every step */
  md_spme* spme;        /* optional reciprocal SPME of the same system, added to the forces (and
                           to energy / virial) every step; NULL = short range only.  The engine's
                           real-space Ewald (md_engine_register_coulomb) completes the split */
} md_sim_params;
enum md_integrator {
  MD_INTEG_LANGEVIN = 0,
  /* the step of ENG/app/lj.nhc-xtc.cu:159-200: COM removal, NoseHoover_Chains2::operator_L(dt/2),
     VelocityVerlet::step1, rebuild check, forces, step2, operator_L(dt/2) */
  MD_INTEG_NHC = 1
};
int md_sim_create(md_sim** out, md_system* sys, md_engine* eng, const md_sim_params* p);
int md_sim_destroy(md_sim* sim);
int md_sim_run(md_sim* sim, int nsteps);
/* number of list rebuilds so far and the last status flags seen on the device */
int md_sim_counters(md_sim* sim, int64_t* steps, int64_t* rebuilds, int* device_flags);
/* 1 when the step graph skips the rebuild chain with a device-side conditional node */
int md_sim_uses_conditional_graph(md_sim* sim, int* out);
/* How a step decides on the device whether to rebuild the cell and neighbour
   lists (the reference decides on the host after reading the displacement
   back, ENG/app/lj.nhc-xtc.cu:193-205):
     MD_REBUILD_FUSED        one cooperative kernel (cell sort, per-slot types,
                             list build) that returns at once unless the
                             device's rebuild flag is set; used whenever the
                             device supports cooperative launches and the
                             system has no bonded topology
     MD_REBUILD_CONDITIONAL  the chain of kernels under a conditional node of
                             the step graph
     MD_REBUILD_GATED        the chain of kernels, each returning at once
                             unless the flag is set (no graph) */
enum { MD_REBUILD_GATED = 0, MD_REBUILD_CONDITIONAL = 1, MD_REBUILD_FUSED = 2 };
int md_sim_rebuild_kind(md_sim* sim, int* out);
/* MD_REBUILD_FUSED (the default, where the device can) or
   MD_REBUILD_CONDITIONAL: the chain of kernels, under a conditional node when
   the step is a graph (gated launches otherwise).  Both give the same lists
   and trajectories bit for bit. */
int md_sim_set_rebuild_kind(md_sim* sim, int kind);
/* A check of the fused rebuild's grid barrier (no counterpart in the
   reference): one cooperative launch of a block per SM meets one barrier on
   the system's state; with skip_block >= 0 that block never arrives, so the
   others give up after limit_s (0 < limit_s <= 10), set the timeout flag and
   return.  *timed_out reports the flag; the call then clears it and
   realigns the barrier counter, so the system stays usable.  Blocks the
   system's stream. */
int md_check_grid_barrier(md_system* sys, int skip_block, double limit_s, int* timed_out);
/* MD_INTEG_NHC runs: md_nhc_get_state of the driver's chain (after the pending
   start-of-step half of the next step) */
int md_sim_get_nhc_state(md_sim* sim, double out[5]);

/* ------------------------------------------------------------ adaptive cutoff
 * Replaces DensityProfile_PiecewiseConst (ENG/src/DensityProfile.cu:27-99),
 * AdaptRCut (ENG/include/AdaptRCut.h:29-107, ENG/src/AdaptRCut.cu:96-508) and
 * PressureCorrection (ENG/src/PressureCorrection.cu:27-340), FP64 on the GPU.
 * Bins: unsigned(L_d/refh) made odd; cutoffs rcmin:rcstep:rcmax. */
typedef struct md_adapt_rcut md_adapt_rcut;
int md_arc_create(md_adapt_rcut** out, md_system* sys, double refh, double rcmin, double rcmax,
                  double rcstep);
int md_arc_destroy(md_adapt_rcut* arc);
int md_arc_get_dims(md_adapt_rcut* arc, int n[3], int* nrc);
/* DensityProfile::deposite of the current coordinates / clearData */
int md_arc_deposit(md_adapt_rcut* arc, md_system* sys);
int md_arc_clear_profile(md_adapt_rcut* arc);
/* use an explicit density profile [nx][ny][nz] instead of deposited samples */
int md_arc_set_profile(md_adapt_rcut* arc, const double* rho);
int md_arc_get_profile(md_adapt_rcut* arc, double* rho);
/* DensityProfile::calculate + AdaptRCut::calError + calRCut(prec) + refineRCut x nrefine
   + PressureCorrection::correction, all on the device */
int md_arc_update(md_adapt_rcut* arc, double prec, int nrefine);
int md_arc_get_error(md_adapt_rcut* arc, double* error /* [nrc][nele] */);
int md_arc_get_rcut(md_adapt_rcut* arc, double* rcut, int* index, double* result_error);
/* k-space kernels: s1k [nrc][nele], s2k [3][nrc][nele] (imaginary parts),
   pressure-correction kernels [3][nrc][nele] */
int md_arc_get_tables(md_adapt_rcut* arc, double* s1k, double* s2k, double* pck);
/* AssignRCut::getRCut + assign: lattice to the system, list rebuild at the next step */
int md_arc_assign(md_adapt_rcut* arc, md_system* sys);
/* tail pressure tensor into MD_STAT_PRESSURE_CORR_*; out (nullable) gets it too */
int md_arc_pressure_correction(md_adapt_rcut* arc, md_system* sys, double out[3]);
/* the reference's schedule inside md_sim_run: deposit every sample_every steps,
   update + assign + pressure correction every update_every steps */
int md_sim_attach_adapt_rcut(md_sim* sim, md_adapt_rcut* arc, int sample_every, int update_every,
                             double prec, int nrefine);

/* ------------------------------------------------- long-range force correction
 * LFC of the fcorr simulation tools (FCR = shortRange.inhomo/template/tools/simulation.fcorr):
 * ForceCorr::reinit(rc, dp) (FCR/src/ForceCorr.cu:112-148, makeS2k :193-262) on the density
 * bins of DensityProfile_PiecewiseConst(box, refh) (odd counts); calError (:150-179) turns
 * the averaged profile into a per-bin correction force field, FFT-convolved in FP64 on the
 * device; AssignForceCorr::getForceCorr / zero / assign (FCR/src/AssignForceCorr.cu:55-178)
 * give every atom the field value of its bin, which the non-bonded kernel adds to the
 * atom's force (FCR/src/InteractionEngine_interface.cu:1118) once the correction is set on
 * the engine.  The field starts at zero (the app's afc.zero()). */
typedef struct md_fcorr md_fcorr;
int md_fcorr_create(md_fcorr** out, md_system* sys, double rc, double refh);
int md_fcorr_destroy(md_fcorr* fc);
int md_fcorr_get_dims(md_fcorr* fc, int n[3]);
/* DensityProfile_PiecewiseConst::deposite / clearData, or an explicit profile [nx][ny][nz] */
int md_fcorr_deposit(md_fcorr* fc, md_system* sys);
int md_fcorr_clear_profile(md_fcorr* fc);
int md_fcorr_set_profile(md_fcorr* fc, const double* rho);
/* the profile of the last update (or the one set) */
int md_fcorr_get_profile(md_fcorr* fc, double* rho);
/* DensityProfile::calculate + ForceCorr::calError + AssignForceCorr::getForceCorr */
int md_fcorr_update(md_fcorr* fc);
/* AssignForceCorr::zero: the per-bin field set to zero */
int md_fcorr_zero(md_fcorr* fc);
/* the field error2r{x,y,z}: real parts re[3][nele], imaginary parts im[3][nele] */
int md_fcorr_get_field(md_fcorr* fc, double* re, double* im);
/* AssignForceCorr::assign: each atom's value from the current field; and the
   per-atom values [N][3] in the caller's atom order */
int md_fcorr_assign(md_fcorr* fc, md_system* sys);
int md_fcorr_get_values(md_fcorr* fc, double* values);
/* the non-bonded kernel adds the per-atom values to the forces (NULL: none) */
int md_engine_set_force_correction(md_engine* eng, md_fcorr* fc);
/* the driver on the fcorr app's schedule (FCR/app/lj.nhc-xtc.cu:172-227): after step i,
   assign when i % assign_every == 0; deposit when (i+1) % sample_every == 0; update
   and clear the samples when (i+1) % update_every == 0.  Also sets it on the engine. */
int md_sim_attach_force_corr(md_sim* sim, md_fcorr* fc, int assign_every, int sample_every, int update_every);
/* Per-step statistics without host involvement: after every step of md_sim_run the
   device writes the MD_STAT_COUNT slots into row (k mod rows) of the host array
   host[rows][MD_STAT_COUNT], k counting the steps since this call.  Page-locked memory is
   used in place; other host memory is registered here.  The rows are valid after
   md_system_synchronize; rows = 0 detaches.  (MDStatistic::updateHost of every step,
   for callers that read each step's energy and virial.) */
int md_sim_set_stats_ring(md_sim* sim, double* host, int rows);

/* ------------------------------------------------------------ synthetic inputs
 * Seeded generators of the benchmark systems (host only, no GPU needed).  The
 * reference builds inputs with gen.conf* tools
 * (shortRange.inhomo/template/tools/gen.conf.tube/app/gen.liquid.cpp). */
/* fcc lattice of nx*ny*nz cubic cells filling box, +-jitter uniform noise */
int md_synth_fcc(int nx, int ny, int nz, const double box[3], double jitter, uint64_t seed,
                 double* pos);
/* random sequential addition, n_in atoms inside |x_axis - center| < half_width,
   the rest outside, all pairs >= min_sep apart */
int md_synth_slab(int n, int n_in, const double box[3], int axis, double center,
                  double half_width, double min_sep, uint64_t seed, double* pos);
/* Maxwell-Boltzmann velocities at temperature (k_B = 1), centre of mass removed */
int md_synth_maxwell(int n, const double* mass, double temperature, uint64_t seed, double* vel);
/* n/2 charges +1 and n/2 charges -1 in seeded random order */
int md_synth_charges(int n, uint64_t seed, double* q);

/* ------------------------------------------------------------ SPME with a Hermite basis
 * ik-SPME whose interpolation basis is optiBasis's symmetric piecewise cubic Hermite basis
 * (optiBasis/Hermite.py:6-130, optiBasis/HatComput.py:155-300: value 1 and slope 0 at 0,
 * coefficients [v_1..v_n, d_1..d_n] at the knots j CC/nbin, n = nbin or nbin - 1 when
 * bound0), in place of the B-spline of ElectrostaticInteraction_rec_BSpline
 * (RE/src/EleRecBSpline.cpp:393-536, the interpolation factor of calB :729-796 taken from
 * the basis' integer samples), with hand-written adjoints for the optiBasis gradient loop
 * (optiBasis/compute_basis.py:38-111).  FP64.  Every array argument is DEVICE memory in the
 * caller's atom order (raw pointers, e.g. torch tensors' data_ptr()), every call is
 * asynchronous on `stream` (NULL: the default stream); coeffs [C][ncoef] is a batch of
 * candidate bases.  For one system of natoms charges on mesh K in box L, splitting beta. */
typedef struct md_hspme md_hspme;
int md_hspme_create(md_hspme** out, int natoms, const int K[3], const double L[3], double beta, double CC,
                    int nbin, int bound0, int device);
int md_hspme_destroy(md_hspme* h);
int md_hspme_num_coeffs(md_hspme* h, int* out);
/* reciprocal energy[C] of charges q [N] at positions r [N][3] for each candidate, and when
   non-NULL: ik forces [C][N][3], dE/dq [C][N], dE/dr [C][N][3] (the exact gradient), dE/dc
   [C][ncoef] */
int md_hspme_energy(md_hspme* h, const double* q, const double* r, const double* coeffs, int C,
                    double* energy, double* forces, double* dE_dq, double* dE_dr, double* dE_dc, void* stream);
/* force-error functional loss[C] = 1/N sum_i |F_i - fref_i|^2 of the ik forces against given
   reference forces fref [N][3] (e.g. md_ewald_exact), and when non-NULL its gradients dL/dq
   [C][N], dL/dr [C][N][3], dL/dc [C][ncoef] (second adjoint of the SPME chain) */
int md_hspme_force_error(md_hspme* h, const double* q, const double* r, const double* coeffs, int C,
                         const double* fref, double* loss, double* dL_dq, double* dL_dr, double* dL_dc,
                         void* stream);

/* ------------------------------------------------------------ optiBasis error functional
 * Replaces HermiteLossFunc / HermiteLossFunc_Bound0 .value / .deriv
 * (optiBasis/IkError.py:166-260) with IkError.prepare_sum / prepare_sum_deriv /
 * estimate / estimate_deriv (optiBasis/IkError.py:32-136) and the hats of
 * HermiteBasisHatComput_Norm1(_Bound0) (optiBasis/HatComput.py:155-300), FP64 on the GPU.
 * Interpolation basis: symmetric piecewise cubic Hermite on nbin bins of [0, CC] (grid
 * units), value 1 and slope 0 at 0; coefficients [v_1..v_n, d_1..d_n] with n = nbin, or
 * n = nbin - 1 when bound0 (the basis vanishes at CC).  Mesh K, rectangular box L,
 * splitting beta, aliasing sum |l| <= l_cut; over_smpl 0 = int(400 nbin / CC).
 * q2 = sum of squared charges and natoms set the scale of the estimate. */
typedef struct md_ikerr md_ikerr;
int md_ikerr_create(md_ikerr** out, const int K[3], const double L[3], double beta, double CC,
                    int nbin, int l_cut, int bound0, int over_smpl, double q2, double natoms,
                    int device);
int md_ikerr_destroy(md_ikerr* h);
int md_ikerr_num_coeffs(md_ikerr* h, int* out);
/* estimate (value) and its gradient for C candidate coefficient vectors coeffs[C][n];
   grads[C][n] may be NULL.  Host arrays; synchronises. */
int md_ikerr_evaluate(md_ikerr* h, int C, const double* coeffs, double* values, double* grads);
/* the same on device arrays, asynchronous on `stream` (NULL = the handle's stream) */
int md_ikerr_evaluate_device(md_ikerr* h, int C, const double* d_coeffs, double* d_values,
                             double* d_grads, void* stream);
/* basis hats along axis d at k = 0..K_d/2 + l_cut K_d: hat0[k] (knot 0) and hats[n][k] */
int md_ikerr_get_hats(md_ikerr* h, int d, double* hat0, double* hats);
/* W_d(m), m = -K_d/2..K_d/2: sum over the other two mesh indices of 2|G(m)|^2 */
int md_ikerr_get_weights(md_ikerr* h, int d, double* W);

#ifdef __cplusplus
}
#endif
#endif
