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
  MD_ERR_NOMEM = 14
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
/* cudaStream_t passed as void*; NULL = the library's own stream. */
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
int md_system_get_box(md_system* sys, double box[3]);
int md_system_set_box(md_system* sys, const double box[3]);
/* per-atom cutoff rcut_i in original order (MDSystem ddata.rcut) */
int md_system_set_rcut(md_system* sys, const float* rcut);
int md_system_get_rcut(md_system* sys, float* rcut);
/* Wrap every atom into [0,L) and update its image counters
   (normalizeSystem, ENG/src/BoxGeometry.cu:6-50). */
int md_system_normalize(md_system* sys);
/* FP64 statistic slots (MDStatistic::updateHost); out has MD_STAT_COUNT entries. */
int md_system_read_stats(md_system* sys, double* out);
int md_system_clear_stats(md_system* sys);

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
/* registBondedInteraction: bonds, angles and exclusions are not part of this path;
   returns MD_OK for n_bonds == 0 and MD_ERR_UNSUPPORTED otherwise. */
int md_engine_register_bonded(md_engine* eng, int n_bonds);
int md_engine_clear_forces(md_engine* eng, md_system* sys);
/* with_stats != 0 accumulates energy and diagonal virial into the FP64 slots. */
int md_engine_apply_nonbonded(md_engine* eng, md_system* sys, md_nlist* nl, int with_stats);
/* applyBondedInteraction: MD_OK with nothing to do when no bonds are registered. */
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
/* the charge mesh Q of the last apply (calQ), [K0][K1][K2] */
int md_spme_get_mesh(md_spme* spme, double* Q);
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
 * (larger ones give MD_ERR_BADARG); the first call on a device looks the array up
 * and should come before any stream capture; calls that overlap in time on one
 * device race on the shared scratch. */
int md_error_estimate_spme_ik_noalloc(md_system* sys, const int K[3], int order, double beta, double* err);
/* splitting beta whose real-space estimate equals target at cutoff rcut */
int md_choose_beta(md_system* sys, double rcut, double target, double* beta);

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
} md_sim_params;
int md_sim_create(md_sim** out, md_system* sys, md_engine* eng, const md_sim_params* p);
int md_sim_destroy(md_sim* sim);
int md_sim_run(md_sim* sim, int nsteps);
/* number of list rebuilds so far and the last status flags seen on the device */
int md_sim_counters(md_sim* sim, int64_t* steps, int64_t* rebuilds, int* device_flags);
/* 1 when the step graph skips the rebuild chain with a device-side conditional node */
int md_sim_uses_conditional_graph(md_sim* sim, int* out);

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

#ifdef __cplusplus
}
#endif
#endif
