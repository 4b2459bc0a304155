// Simulation driver: the hot loop of ENG/app/lj.nhc-xtc.cu:159-274 for the
// Langevin path, with the rebuild decision taken on the device.
//
// One step, recorded once as a CUDA graph of kernel nodes:
//   k_lv_step1   particle B A O A, displacement test; its last block writes
//                the rebuild decision into a graph conditional
//   IF(rebuild)  bin, scan, scatter, order, gather, copy back, list build
//   LJ           forces (overwrite) + FP64 energy / virial (store)
//   SPME         (when attached) the reciprocal chain; with the Langevin
//                integrator a second branch beside LJ, joined by k_lv_step2
//   k_lv_step2   closing B (adding the SPME forces, energy and virial),
//                kinetic tensor, pressure, box momentum half kick, and the
//                box B A O A of the next step
// Where the driver cannot create conditional nodes the rebuild kernels are
// recorded unconditionally and return at once unless the device flag is set.
// Density sampling and the adaptive-cutoff update run between graph launches
// on the same stream on the reference's schedule (every 40 / 2000 steps).
#include <cmath>
#include <cstring>
#include <vector>
#include "device_common.cuh"

struct md_adapt_rcut;
extern "C" int md_arc_deposit(md_adapt_rcut* a, md_system* sys);
extern "C" int md_arc_update(md_adapt_rcut* a, double prec, int nrefine);
extern "C" int md_arc_assign(md_adapt_rcut* a, md_system* sys);
extern "C" int md_arc_pressure_correction(md_adapt_rcut* a, md_system* sys, double out[3]);
extern "C" int md_arc_clear_profile(md_adapt_rcut* a);

struct md_sim {
  md_system* sys = nullptr;
  md_engine* eng = nullptr;
  md_sim_params p;
  md_cell_list* cl = nullptr;
  md_nlist* nl = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // MD_SIM_MULTI consecutive steps in one graph, launched when no host-side
  // work (density samples, cutoff or correction updates) falls between them
  cudaGraph_t graph_multi = nullptr;
  cudaGraphExec_t exec_multi = nullptr;
  bool conditional = false;
  bool fused = false;  // the rebuild is the flag-gated cooperative kernel
  bool allow_fused = true;  // md_sim_set_rebuild_kind
  float* lattice_in_graph = nullptr;
  int topo_in_graph = -1;
  int64_t steps = 0;
  md_nhc* nhc = nullptr;  // MD_INTEG_NHC
  bool nhc_settled = false;  // velocities / chain brought to the end of the last step
  // long-range force correction schedule
  md_fcorr* fcorr = nullptr;
  int fc_assign_every = 0, fc_sample_every = 0, fc_update_every = 0;
  // adaptive cutoff schedule
  md_adapt_rcut* arc = nullptr;
  int sample_every = 0, update_every = 0, nrefine = 0;
  double prec = 0;
  // statistics ring in page-locked host memory: each step's slots are written
  // there by the device, row (count mod rows)
  double* ring = nullptr;     // device view of the host rows
  int ring_rows = 0;
  unsigned* ring_count = nullptr;
  void* ring_registered = nullptr;  // host pointer this library registered
};

static void ring_release(md_sim* s);

// steps per multi-step graph: a graph launch costs a few microseconds that a
// step of tens of microseconds would otherwise pay each time
constexpr int MD_SIM_MULTI = 8;

// the step's statistic slots into the next row of the host ring
__global__ void k_stats_ring(const DevState* st, double* ring, int rows, unsigned* count) {
  const unsigned r = *count;
  const int t = threadIdx.x;
  if (t < MD_STAT_COUNT) ring[(size_t)(r % (unsigned)rows) * MD_STAT_COUNT + t] = st->stats[t];
  __syncthreads();
  if (t == 0) *count = r + 1;
}

static int record_step(md_sim* s, Recorder* rec, bool use_graph) {
  md_system* sys = s->sys;
  cudaGraphConditionalHandle h = 0;
  bool cond = false;
  // the rebuild as one flag-gated cooperative kernel where the device can
  // run it, else the chain of kernels under a conditional node (or gated)
  const bool fused = s->allow_fused && rebuild_fused_ok(sys, s->nl);
  if (use_graph && rec->graph && !fused) {
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, rec->graph, 0, 0);
    cond = (e == cudaSuccess);
    if (!cond) cudaGetLastError();
  }
  const bool nhc = s->nhc != nullptr;
  if (fused && !nhc) {
    // the Langevin first half and the rebuild in one kernel
    if (int r = rebuild_fused_impl(s->cl, s->nl, sys, rec, true)) return r;
  } else if (nhc) {
    if (int r = nhc_vv1_impl(s->nhc, s->nl, s->p.lv.dt, rec, h, cond ? 1 : 0)) return r;
  } else {
    if (int r = langevin_step1_impl(sys, s->nl, rec, false, h, cond ? 1 : 0)) return r;
  }
  if (fused && nhc) {
    if (int r = rebuild_fused_impl(s->cl, s->nl, sys, rec, false)) return r;
  } else if (fused) {
  } else if (cond) {
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    MD_CUDA(cudaGraphAddNode(&node, rec->graph, &rec->last, 1, &cp));
    Recorder body;
    body.graph = cp.conditional.phGraph_out[0];
    body.stream = rec->stream;
    if (int r = cells_rebuild_impl(s->cl, sys, &body, false)) return r;
    if (int r = nlist_build_impl(s->nl, sys, s->cl, &body, false)) return r;
    rec->last = node;
    rec->has_last = true;
  } else {
    if (int r = cells_rebuild_impl(s->cl, sys, rec, true)) return r;
    if (int r = nlist_build_impl(s->nl, sys, s->cl, rec, true)) return r;
  }
  s->conditional = cond;
  s->fused = fused;
  // Langevin with SPME: the reciprocal chain is a second branch beside the
  // real-space kernel (both depend on the rebuild); it stores its forces in
  // its own buffer and leaves its energy and virial for the closing kick,
  // which adds both in
  const bool branch = s->p.spme && !nhc;
  const cudaGraphNode_t fork = rec->last;
  const bool fork_has = rec->has_last;
  // the Langevin closing kick adds up the non-bonded statistics rows itself
  // when nothing else adds to those slots in between (no bonded terms)
  const bool defer = !nhc && !topo_has_terms(sys->topo);
  if (int r = lj_apply_impl(s->eng, sys, s->nl, true, true, rec, !defer)) return r;
  if (int r = bonded_apply_impl(sys, rec, 1)) return r;
  if (s->p.spme) {
    const cudaGraphNode_t lj = rec->last;
    if (branch && rec->graph) {
      rec->last = fork;
      rec->has_last = fork_has;
    }
    if (int r = spme_apply_impl(s->p.spme, true, rec, branch)) return r;
    if (branch && rec->graph) rec->join = lj;
  }
  if (nhc) {
    // closing kick + operator_L(dt/2), then this step's successor's COM
    // removal and operator_L(dt/2), as a pending velocity map
    if (int r = nhc_vv2_impl(s->nhc, s->p.lv.dt, rec, 1, 1, 1, 1)) return r;
  } else {
    if (int r = langevin_step2_impl(sys, rec, 1, 1, branch ? spme_force_buffer(s->p.spme) : nullptr, branch ? 1 : 0,
                                    defer ? lj_stat_rows(sys) : 0, 1))
      return r;
  }
  if (s->ring) {
    DevState* st = sys->st;
    void* a[] = {&st, &s->ring, &s->ring_rows, &s->ring_count};
    if (int r = rec_launch(rec, (const void*)k_stats_ring, dim3(1), dim3(32), 0, a)) return r;
  }
  return MD_OK;
}

static void release_graphs(md_sim* s) {
  if (s->exec) { cudaGraphExecDestroy(s->exec); s->exec = nullptr; }
  if (s->graph) { cudaGraphDestroy(s->graph); s->graph = nullptr; }
  if (s->exec_multi) { cudaGraphExecDestroy(s->exec_multi); s->exec_multi = nullptr; }
  if (s->graph_multi) { cudaGraphDestroy(s->graph_multi); s->graph_multi = nullptr; }
}

static int build_graph(md_sim* s) {
  release_graphs(s);
  MD_CUDA(cudaGraphCreate(&s->graph, 0));
  // the grid barrier's counter stays aligned unless a wait gave up: start clean
  MD_CUDA(cudaMemsetAsync(&s->sys->st->gbar, 0, sizeof(unsigned long long), s->sys->stream));
  Recorder g;
  g.graph = s->graph;
  g.stream = s->sys->stream;
  if (int r = record_step(s, &g, true)) return r;
  MD_CUDA(cudaGraphInstantiate(&s->exec, s->graph, 0));
  // the same step recorded MD_SIM_MULTI times in a row
  MD_CUDA(cudaGraphCreate(&s->graph_multi, 0));
  Recorder m;
  m.graph = s->graph_multi;
  m.stream = s->sys->stream;
  for (int k = 0; k < MD_SIM_MULTI; ++k)
    if (int r = record_step(s, &m, true)) return r;
  MD_CUDA(cudaGraphInstantiate(&s->exec_multi, s->graph_multi, 0));
  s->lattice_in_graph = s->sys->d_lattice;
  s->topo_in_graph = s->sys->topo_version;
  return MD_OK;
}

extern "C" int md_sim_destroy(md_sim* s) {
  if (!s) return MD_OK;
  if (s->sys && s->sys->stream) cudaStreamSynchronize(s->sys->stream);
  ring_release(s);
  release_graphs(s);
  md_nlist_destroy(s->nl);
  md_cell_list_destroy(s->cl);
  md_nhc_destroy(s->nhc);
  delete s;
  return MD_OK;
}

extern "C" int md_sim_create(md_sim** out, md_system* sys, md_engine* eng, const md_sim_params* p) {
  if (!out || !sys || !eng || !p || !(p->skin >= 0) || !(p->cell_size > 0)) {
    md_set_error("md_sim_create: bad arguments");
    return MD_ERR_BADARG;
  }
  if (!eng->has_lj) { md_set_error("md_sim_create: register a non-bonded interaction first"); return MD_ERR_BADARG; }
  if (p->spme && !spme_belongs_to(p->spme, sys)) {
    md_set_error("md_sim_create: the SPME object belongs to another system");
    return MD_ERR_BADARG;
  }
  md_sim* s = new md_sim();
  s->sys = sys;
  s->eng = eng;
  s->p = *p;
  int r;
  auto fail = [&](int code) { md_sim_destroy(s); return code; };
  if ((r = md_langevin_setup(sys, &p->lv))) return fail(r);
  if ((r = md_cell_list_create(&s->cl, sys, p->cell_size, 7, 1))) return fail(r);
  // list radius for the capacity estimate: largest rcut + skin
  std::vector<float> rc(sys->N);
  if ((r = md_system_get_rcut(sys, rc.data()))) return fail(r);
  float rmax = 0;
  for (float v : rc) rmax = v > rmax ? v : rmax;
  if (!(rmax > 0)) { md_set_error("md_sim_create: per-atom cutoffs not set"); return fail(MD_ERR_BADARG); }
  if (p->max_rcut > rmax) rmax = (float)p->max_rcut;
  double rlist = rmax + p->skin;
  if ((r = md_nlist_create(&s->nl, sys, rlist, p->skin, p->expansion > 0 ? p->expansion : 1.0, p->nl_mode))) return fail(r);
  if ((r = md_cell_list_rebuild(s->cl, sys))) return fail(r);
  // capacity: lists of every atom at the largest cutoff the run may assign,
  // 20% + 32 head room (a list that still outgrows it raises the overflow flag)
  {
    std::vector<float> keep(sys->N);
    if ((r = md_system_get_rcut(sys, keep.data()))) return fail(r);
    std::vector<float> big(sys->N, rmax);
    if ((r = md_system_set_rcut(sys, big.data()))) return fail(r);
    if ((r = md_nlist_fit(s->nl, sys, s->cl))) return fail(r);
    DevState hs;
    if ((r = sys->read_state(hs))) return fail(r);
    if ((r = md_system_set_rcut(sys, keep.data()))) return fail(r);
    int want = ((int)(hs.max_nnb * 1.2) + 32 + 31) & ~31;
    if (want > s->nl->cap) {
      cudaFree(s->nl->list);
      s->nl->list = nullptr;
      s->nl->cap = want;
      if (cudaMalloc(&s->nl->list, sizeof(int) * (size_t)want * sys->N) != cudaSuccess) return fail(md_cuda_fail(cudaGetLastError(), "nlist realloc"));
    }
    if ((r = md_nlist_rebuild(s->nl, sys, s->cl))) return fail(r);
  }
  // initial forces, pressure and the box move of the first step
  Recorder rec;
  rec.stream = sys->stream;
  if ((r = lj_apply_impl(eng, sys, s->nl, true, true, &rec))) return fail(r);
  if (p->spme && (r = spme_apply_impl(p->spme, true, &rec))) return fail(r);
  if (p->integrator == MD_INTEG_NHC) {
    if (!(p->nhc_tau > 0)) { md_set_error("md_sim_create: the Nose-Hoover chain needs nhc_tau > 0"); return fail(MD_ERR_BADARG); }
    if ((r = md_nhc_create(&s->nhc, sys, p->lv.temperature, p->nhc_tau, p->remove_com))) return fail(r);
    // step 0 opens with COM removal and operator_L(dt/2): pending velocity map
    if ((r = nhc_vv2_impl(s->nhc, p->lv.dt, &rec, 0, 0, 1, 1))) return fail(r);
  } else if (p->integrator != MD_INTEG_LANGEVIN) {
    md_set_error("md_sim_create: unknown integrator %d", p->integrator);
    return fail(MD_ERR_BADARG);
  } else if ((r = langevin_step2_impl(sys, &rec, 0, 1))) {
    return fail(r);
  }
  // the fused rebuild's grid barrier counter starts clean (build_graph does
  // it again whenever it records the step)
  MD_CUDA(cudaMemsetAsync(&sys->st->gbar, 0, sizeof(unsigned long long), sys->stream));
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  if (p->use_graph)
    if ((r = build_graph(s))) return fail(r);
  *out = s;
  return MD_OK;
}

static void ring_release(md_sim* s) {
  if (s->ring_count) cudaFree(s->ring_count);
  if (s->ring_registered) cudaHostUnregister(s->ring_registered);
  s->ring = nullptr;
  s->ring_rows = 0;
  s->ring_count = nullptr;
  s->ring_registered = nullptr;
}

extern "C" int md_sim_set_stats_ring(md_sim* s, double* host, int rows) {
  if (!s || rows < 0 || (rows > 0 && !host)) return MD_ERR_BADARG;
  MD_CUDA(cudaStreamSynchronize(s->sys->stream));
  ring_release(s);
  if (rows > 0) {
    // page-locked memory is device-addressable under unified addressing; other
    // host memory is registered (and unregistered again by this library)
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, host) != cudaSuccess || at.type != cudaMemoryTypeHost) {
      cudaGetLastError();
      MD_CUDA(cudaHostRegister(host, sizeof(double) * MD_STAT_COUNT * (size_t)rows, cudaHostRegisterMapped));
      s->ring_registered = host;
    }
    double* dev = nullptr;
    MD_CUDA(cudaHostGetDevicePointer((void**)&dev, host, 0));
    MD_CUDA(cudaMalloc(&s->ring_count, sizeof(unsigned)));
    // ordered with the step graphs, which run on the system's (non-blocking) stream
    MD_CUDA(cudaMemsetAsync(s->ring_count, 0, sizeof(unsigned), s->sys->stream));
    s->ring = dev;
    s->ring_rows = rows;
  }
  if (s->exec)
    if (int r = build_graph(s)) return r;
  return MD_OK;
}

extern "C" int md_sim_attach_force_corr(md_sim* s, md_fcorr* fc, int assign_every, int sample_every,
                                        int update_every) {
  if (!s || !fc || assign_every < 1 || sample_every < 1 || update_every < 1) {
    md_set_error("md_sim_attach_force_corr: bad arguments");
    return MD_ERR_BADARG;
  }
  s->fcorr = fc;
  s->fc_assign_every = assign_every;
  s->fc_sample_every = sample_every;
  s->fc_update_every = update_every;
  if (int r = md_engine_set_force_correction(s->eng, fc)) return r;
  // the recorded non-bonded kernel must see the correction values
  if (s->exec)
    if (int r = build_graph(s)) return r;
  return MD_OK;
}

extern "C" int md_sim_attach_adapt_rcut(md_sim* s, md_adapt_rcut* arc, int sample_every, int update_every,
                                        double prec, int nrefine) {
  if (!s || !arc || sample_every < 1 || update_every < 1 || !(prec > 0) || nrefine < 0) {
    md_set_error("md_sim_attach_adapt_rcut: bad arguments");
    return MD_ERR_BADARG;
  }
  s->arc = arc;
  s->sample_every = sample_every;
  s->update_every = update_every;
  s->prec = prec;
  s->nrefine = nrefine;
  return MD_OK;
}

// true when host-side work is due after any of the n steps j0 .. j0 + n - 1
// (j = the step's index; the schedules of md_sim_run below)
static bool host_work_within(const md_sim* s, int64_t j0, int n) {
  for (int64_t j = j0; j < j0 + n; ++j) {
    if (s->fcorr && (j % s->fc_assign_every == 0 || (j + 1) % s->fc_sample_every == 0 ||
                     (j + 1) % s->fc_update_every == 0))
      return true;
    if (s->arc && ((j + 1) % s->sample_every == 0 || (j + 1) % s->update_every == 0)) return true;
  }
  return false;
}

extern "C" int md_sim_run(md_sim* s, int nsteps) {
  if (!s || nsteps < 0) return MD_ERR_BADARG;
  md_system* sys = s->sys;
  if (s->exec && (sys->d_lattice != s->lattice_in_graph || sys->topo_version != s->topo_in_graph))
    if (int r = build_graph(s)) return r;
  if (s->nhc && s->nhc_settled && nsteps > 0) {
    // re-open the step the last run closed: COM removal + operator_L(dt/2)
    Recorder rec;
    rec.stream = sys->stream;
    if (int r = nhc_vv2_impl(s->nhc, s->p.lv.dt, &rec, 0, 0, 1, 0)) return r;
    s->nhc_settled = false;
  }
  for (int i = 0; i < nsteps; ++i) {
    if (s->exec_multi && nsteps - i >= MD_SIM_MULTI && !host_work_within(s, s->steps, MD_SIM_MULTI - 1)) {
      // steps s->steps .. s->steps + MD_SIM_MULTI - 1 in one launch; host work
      // due after the last of them runs below as after a single step
      MD_CUDA(cudaGraphLaunch(s->exec_multi, sys->stream));
      s->steps += MD_SIM_MULTI - 1;
      i += MD_SIM_MULTI - 1;
    } else if (s->exec) {
      MD_CUDA(cudaGraphLaunch(s->exec, sys->stream));
    } else {
      Recorder rec;
      rec.stream = sys->stream;
      if (int r = record_step(s, &rec, false)) return r;
    }
    if (s->fcorr) {
      // FCR/app/lj.nhc-xtc.cu:172-227, step i = s->steps: assign after the
      // force of step i, then the samples and the update after step i + 1
      const int64_t i0 = s->steps;
      if (i0 % s->fc_assign_every == 0)
        if (int r = md_fcorr_assign(s->fcorr, sys)) return r;
      if ((i0 + 1) % s->fc_sample_every == 0)
        if (int r = md_fcorr_deposit(s->fcorr, sys)) return r;
      if ((i0 + 1) % s->fc_update_every == 0) {
        if (int r = md_fcorr_update(s->fcorr)) return r;
        if (int r = md_fcorr_clear_profile(s->fcorr)) return r;
      }
    }
    s->steps += 1;
    if (s->arc) {
      // lj.nhc-xtc.cu:226-254: deposit every sample_every steps, new rc map and
      // tail correction every update_every steps
      if (s->steps % s->sample_every == 0)
        if (int r = md_arc_deposit(s->arc, sys)) return r;
      if (s->steps % s->update_every == 0) {
        if (int r = md_arc_update(s->arc, s->prec, s->nrefine)) return r;
        if (int r = md_arc_assign(s->arc, sys)) return r;
        if (int r = md_arc_pressure_correction(s->arc, sys, nullptr)) return r;
        if (int r = md_arc_clear_profile(s->arc)) return r;
        if (s->exec && sys->d_lattice != s->lattice_in_graph)
          if (int r = build_graph(s)) return r;
      }
    }
  }
  if (s->nhc && !s->nhc_settled) {
    // velocities and chain as the reference has them after the last step
    if (int r = nhc_settle_impl(s->nhc)) return r;
    s->nhc_settled = true;
  }
  return MD_OK;
}

extern "C" int md_sim_counters(md_sim* s, int64_t* steps, int64_t* rebuilds, int* flags) {
  if (!s) return MD_ERR_BADARG;
  DevState hs;
  if (int r = s->sys->read_state(hs)) return r;
  if (steps) *steps = s->steps;
  if (rebuilds) *rebuilds = (int64_t)hs.rebuilds;
  if (flags) *flags = (int)hs.flags;
  if (hs.flags & FLAG_NL_OVERFLOW) {
    md_set_error("neighbour list overflow during the run (largest list %d, capacity %d)", hs.max_nnb, s->nl->cap);
    return MD_ERR_NLIST_OVERFLOW;
  }
  if (hs.flags & FLAG_NAN) { md_set_error("non-finite coordinates during the run"); return MD_ERR_BADARG; }
  if (hs.flags & FLAG_TIMEOUT) { md_set_error("a grid barrier of the rebuild gave up waiting"); return MD_ERR_TIMEOUT; }
  return MD_OK;
}

extern "C" int md_sim_get_nhc_state(md_sim* s, double out[5]) {
  if (!s || !out) return MD_ERR_BADARG;
  if (!s->nhc) { md_set_error("md_sim_get_nhc_state: the run does not use the Nose-Hoover chain"); return MD_ERR_BADARG; }
  return md_nhc_get_state(s->nhc, out);
}

extern "C" int md_sim_rebuild_kind(md_sim* s, int* out) {
  if (!s || !out) return MD_ERR_BADARG;
  *out = s->fused ? MD_REBUILD_FUSED : (s->exec && s->conditional) ? MD_REBUILD_CONDITIONAL : MD_REBUILD_GATED;
  return MD_OK;
}

extern "C" int md_sim_set_rebuild_kind(md_sim* s, int kind) {
  if (!s || (kind != MD_REBUILD_FUSED && kind != MD_REBUILD_CONDITIONAL)) {
    md_set_error("md_sim_set_rebuild_kind: MD_REBUILD_FUSED or MD_REBUILD_CONDITIONAL");
    return MD_ERR_BADARG;
  }
  s->allow_fused = kind == MD_REBUILD_FUSED;
  if (s->exec) return build_graph(s);
  s->fused = s->allow_fused && rebuild_fused_ok(s->sys, s->nl);
  return MD_OK;
}

extern "C" int md_sim_uses_conditional_graph(md_sim* s, int* out) {
  if (!s || !out) return MD_ERR_BADARG;
  *out = (s->exec && s->conditional) ? 1 : 0;
  return MD_OK;
}
