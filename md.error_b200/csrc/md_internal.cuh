// Internal declarations shared by the translation units of libmdforce.
// Device data layout (all per-atom arrays in CELL ORDER, slot k):
//   pos[k]   Real4  x,y,z wrapped into the box at the last rebuild, w = charge
//   vel[k]   Real4  vx,vy,vz, w = 1/m
//   force[k] double4 accumulated force (FP64 in both precisions)
//   image[k] int4   periodic image counters (coordNoi{x,y,z})
//   id[k]    int    original atom index
//   rcut[k]  float  per-atom cutoff (AssignRCut lattice value)
// The box, the statistic slots, the rebuild/overflow flags and the barostat
// state live in one device-resident DevState so that a captured step never
// needs a host round trip.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>
#include "../../include/mdforce.h"

struct alignas(32) double4a {
  double x, y, z, w;
};

template <class R> struct V4;
template <> struct V4<float> { typedef float4 T; };
template <> struct V4<double> { typedef double4a T; };

// device flag bits
enum : unsigned {
  FLAG_REBUILD = 1u,        // displacement exceeded skin/2 (or forced)
  FLAG_NL_OVERFLOW = 2u,    // mdErrorShortNeighborList
  FLAG_CELL_INDEX = 4u,     // mdErrorOverFlowCellIdx
  FLAG_NAN = 8u,            // non-finite coordinate met
  FLAG_TIMEOUT = 16u,
  FLAG_FORCE_REBUILD = 32u, // rebuild at the next step (cutoffs or box changed)
  FLAG_QUADRATURE = 64u     // adaptive quadrature hit its depth bound
};

// reduction counters (one per kind of last-block reduction)
enum { RED_LJ = 0, RED_KIN = 1, RED_DISP = 2, RED_SPME = 3, RED_MISC = 4, RED_BOND = 5 /* and 6 */,
       RED_NLWORK = 7 /* home cells handed out by the fused rebuild */, RED_COUNT = 8 };

struct DevState {
  double L[3];       // box edge, FP64 master copy
  double Li[3];      // 1/L
  float Lf[3];       // binary32 box.size (BoxGeometry.h setBoxSize)
  float Lif[3];      // binary32 box.sizei = 1/x computed in float
  double stats[MD_STAT_COUNT];
  unsigned flags;
  unsigned red_counter[RED_COUNT];
  int max_nnb;       // largest list length seen at the last build
  int pad0;
  unsigned long long step;     // Langevin step counter (RNG counter)
  unsigned long long rebuilds; // number of list builds
  double max_disp2;            // last max squared displacement
  // barostat (anisotropic Langevin piston on the box lengths)
  double ph[3];      // box momentum p_h
  double Mh[3];      // box mass
  double lam1[3], lam2[3]; // scale factors of the two A half steps of this step
  double Pcur[3];    // diagonal pressure at the end of the last step
  double scratch[8]; // reduction target of multi-slot sums merged afterwards
  double kick_sums[8]; // closing kick: kinetic tensor and the non-bonded statistics rows
  double Lnext[3];   // box of the next step, committed by that step's first kernel
  double box_xi[4];  // the box normals of the coming step, computed ahead in the closing kick
  int box_pending;
  unsigned ncell_busy;  // home cells of 4 atoms or more listed by the fused rebuild
  unsigned ncell_light; // and of 1 to 3 atoms
  unsigned pad1;
  unsigned long long gbar;  // grid barrier of the fused rebuild (grid_barrier)
};

// host helpers -------------------------------------------------------------
void md_set_error(const char* fmt, ...);
int md_cuda_fail(cudaError_t e, const char* what);
#define MD_CUDA(call)                                   \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return md_cuda_fail(_e, #call); \
  } while (0)
#define MD_CHECK_LAUNCH(what)                           \
  do {                                                  \
    cudaError_t _e = cudaGetLastError();                \
    if (_e != cudaSuccess) return md_cuda_fail(_e, what); \
  } while (0)

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// box update on the host side copy
void box_fill(DevState& s, const double L[3]);

struct md_topo;  // bonded terms and exclusions by atom id (bonded.cu)

struct md_system {
  int N = 0;
  int prec = MD_PREC_MIXED;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  void* pos = nullptr;      // Real4
  void* vel = nullptr;      // Real4
  double4a* force = nullptr;
  int4* image = nullptr;
  int* id = nullptr;
  float* rcut = nullptr;
  // gather targets used by the cell sort
  void* t_pos = nullptr;
  void* t_vel = nullptr;
  double4a* t_force = nullptr;
  int4* t_image = nullptr;
  int* t_id = nullptr;
  float* t_rcut = nullptr;
  DevState* st = nullptr;   // device state
  double* partials = nullptr;  // block partial sums for reductions
  double* nb_rows = nullptr;   // non-bonded statistics, one row of 5 sums per warp
  int max_partial_blocks = 0;
  // pinned host staging
  void* h_stage = nullptr;
  size_t h_stage_bytes = 0;
  // atom types (TypeType of the reference): by original id and by current
  // slot (refreshed by every cell sort); 0 for every atom unless given
  uint8_t* type_by_id = nullptr;
  uint8_t* type = nullptr;
  int ntypes = 1;
  // bonded topology (null when none); the version counts its changes
  md_topo* topo = nullptr;
  int topo_version = 0;
  // rc lattice (AssignRCut)
  float* d_lattice = nullptr;
  int lat_n[3] = {0, 0, 0};
  // Langevin parameters (md_langevin_setup)
  md_langevin_params lv;
  bool lv_set = false;
  size_t real_size() const { return prec == MD_PREC_FP64 ? sizeof(double) : sizeof(float); }
  size_t r4_size() const { return prec == MD_PREC_FP64 ? sizeof(double4a) : sizeof(float4); }
  int read_state(DevState& s);
};

struct md_cell_list {
  int ncell[3] = {1, 1, 1};
  int ntot = 1;
  double cell_size = 0;
  int bdir = 7, divide = 1;
  uint32_t* cell_of = nullptr;     // cell of slot k (after sort: sorted order)
  uint32_t* t_cell = nullptr;      // cell of slot k before the sort
  uint32_t* slot = nullptr;        // rank inside the cell from the atomic count
  uint32_t* count = nullptr;       // atoms per cell
  uint32_t* start = nullptr;       // exclusive scan, ntot+1
  uint32_t* members = nullptr;     // cell member lists (current index)
  uint32_t* perm = nullptr;        // perm[new] = old
  // the slots of each cell ordered by z: zord[start[c] .. start[c+1]) (the list
  // build reads runs of cells in this order to cut each atom's z window exactly)
  uint32_t* zord = nullptr;
  uint32_t* busy = nullptr;        // the fused rebuild's non-empty cells: the fuller ones from the front, the rest from the back
  bool built = false;
};

// Row layout of the neighbour list: rows hold cap entries (a multiple of 32)
// in 32-entry lines, each line stored transposed 8 x 4 so that a force
// kernel with 8 lanes per atom reads one 16-byte vector per lane per line
// and lane l holds the line's logical entries l, l+8, l+16, l+24 (the 8
// lanes then gather 8 consecutive neighbours at a time).  Logical entry e of
// a row sits at nl_slot(e).
__host__ __device__ __forceinline__ int nl_slot(int e) {
  return (e & ~31) | ((e & 7) << 2) | ((e >> 3) & 3);
}

struct md_nlist {
  double rlist = 0, skin = 0, expansion = 1;
  int mode = MD_NL_MINIMAGE;
  int cap = 0;
  int N = 0;
  int* list = nullptr;    // [N][cap] row-major (slot indices)
  int* nnb = nullptr;     // [N]
  void* backup = nullptr; // Real4 positions at the last build
  bool built = false;
};

struct md_engine {
  md_system* sys = nullptr;
  bool has_lj = false;
  double eps = 1, sigma = 1, shift = 0;
  // per type pair LJ (SystemNonBondedInteraction::add / AtomNBForceTable):
  // nt > 0 selects the typed kernels; pairs not given take no force
  int nt = 0;
  int nb_kind[16][16] = {};        // md_nb_kind per type pair (symmetric), 0: none
  double nb_param[16][16][6] = {};  // the kind's user parameters
  void* d_tab = nullptr;            // float4 [3*16*16] then double4a [3*16*16]
  bool tab_dirty = false;
  bool has_coul = false;
  double beta = 0;
  int n_bonds = 0;
  md_fcorr* fcorr = nullptr;  // long-range force correction added by the non-bonded kernel
};
// per-atom correction values (by atom id) of an md_fcorr
const double4a* fcorr_values(const md_fcorr* f);

// launch helper: direct launch or kernel-node recording ---------------------
struct Recorder {
  cudaGraph_t graph = nullptr;   // when non-null, launches become kernel nodes
  cudaGraphNode_t last = nullptr;
  bool has_last = false;
  cudaGraphNode_t join = nullptr;  // second dependency of the next node (a branch joining back)
  cudaStream_t stream = nullptr;
};
int rec_launch(Recorder* r, const void* func, dim3 grid, dim3 block, size_t smem, void** args);
// the same as a cooperative launch (every block resident at once)
int rec_launch_coop(Recorder* r, const void* func, dim3 grid, dim3 block, size_t smem, void** args);

// kernels entry points implemented in the .cu files -------------------------
int cells_rebuild_impl(md_cell_list* cl, md_system* sys, Recorder* rec, bool conditional);
int nlist_build_impl(md_nlist* nl, md_system* sys, md_cell_list* cl, Recorder* rec, bool conditional);
// The cell sort, the per-slot types and the list build as one cooperative
// kernel that returns at once unless the device's rebuild flag is set (no
// bonded topology: its slot map and exclusions stay separate kernels).
// with_lv: the same kernel opens with the Langevin particle B A O A and the
// displacement test of k_lv_step1, whose work it replaces.
// rebuild_fused_ok tells whether the device can run it for this system.
bool rebuild_fused_ok(const md_system* sys, const md_nlist* nl);
int rebuild_fused_impl(md_cell_list* cl, md_nlist* nl, md_system* sys, Recorder* rec, bool with_lv);
int lj_apply_impl(md_engine* eng, md_system* sys, md_nlist* nl, bool with_stats, bool overwrite, Recorder* rec,
                  bool finish_stats = true);
int lj_stat_rows(const md_system* sys);
// bonded terms (bonded.cu): slot map refresh after a cell sort, exclusion pass
// after a list build, the bonded force kernel; each a no-op without topology
void topo_destroy(md_topo* t);
bool topo_has_terms(const md_topo* t);
int topo_slot_launch(md_system* sys, Recorder* rec, bool gated);
// per-slot atom types from the per-id ones after a sort (system.cu)
int types_slot_launch(md_system* sys, Recorder* rec, bool gated);
constexpr int MD_MAX_TYPES = 16;
int topo_exclude_launch(md_system* sys, md_nlist* nl, Recorder* rec, bool gated);
int bonded_apply_impl(md_system* sys, Recorder* rec, int with_stats);
int langevin_step1_impl(md_system* sys, md_nlist* nl, Recorder* rec, bool with_box_kernel,
                        cudaGraphConditionalHandle cond, int use_cond);
// fadd: per-atom force of a concurrent branch (SPME), added into the force
// array by the closing kick; merge_rec: the branch's reciprocal energy and
// virial (DevState::scratch) are merged into the statistics by its last block;
// nb_rows > 0: the non-bonded statistics rows left in sys->nb_rows
// (lj_apply_impl without finish_stats) are added up by the kick, stored into
// their slots with nb_store, else added
int langevin_step2_impl(md_system* sys, Recorder* rec, int kick, int advance, const double4a* fadd = nullptr,
                        int merge_rec = 0, int nb_rows = 0, int nb_store = 0);
int clear_stats_impl(md_system* sys, Recorder* rec, int first, int count);
int nhc_vv1_impl(md_nhc* h, md_nlist* nl, double dt, Recorder* rec, cudaGraphConditionalHandle cond,
                 int use_cond);
int nhc_vv2_impl(md_nhc* h, double dt, Recorder* rec, int kick, int end, int start, int account);
int nhc_settle_impl(md_nhc* h);
// concurrent: the chain may run beside the real-space kernel; it then stores
// its forces in spme_force_buffer() and leaves its energy and virial in
// DevState::scratch for the closing kick to merge
int spme_apply_impl(md_spme* s, bool with_stats, Recorder* rec, bool concurrent = false);
const double4a* spme_force_buffer(const md_spme* s);
bool spme_belongs_to(const md_spme* s, const md_system* sys);
int set_flag_impl(md_system* sys, unsigned bits, Recorder* rec);
