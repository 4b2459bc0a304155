// Simulation driver: the hot loop of ENG/app/lj.nhc-xtc.cu:159-274 for the
// Langevin path, with the rebuild decision taken on the device.
// One step = k_lv_box, k_lv_step1 (B A O A + displacement flag), the gated
// rebuild chain (bin, scan, scatter, order, gather, copy back, list build),
// stats clear, LJ (overwrite, +stats), k_lv_step2 (B, kinetic tensor,
// pressure, box half kick).  The step is recorded once as a CUDA graph of
// kernel nodes and replayed; gated kernels return at once when the device
// flag says no rebuild is due.
#include <cmath>
#include <cstring>
#include <vector>
#include "device_common.cuh"

struct md_sim {
  md_system* sys = nullptr;
  md_engine* eng = nullptr;
  md_sim_params p;
  md_cell_list* cl = nullptr;
  md_nlist* nl = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t steps = 0;
};

static int record_step(md_sim* s, Recorder* rec) {
  md_system* sys = s->sys;
  bool stats = true;
  if (int r = langevin_step1_impl(sys, s->nl, rec)) return r;
  if (int r = cells_rebuild_impl(s->cl, sys, rec, true)) return r;
  if (int r = nlist_build_impl(s->nl, sys, s->cl, rec, true)) return r;
  if (int r = clear_stats_impl(sys, rec, MD_STAT_NB_ENERGY, 4)) return r;
  if (int r = lj_apply_impl(s->eng, sys, s->nl, stats, true, rec)) return r;
  if (int r = langevin_step2_impl(sys, rec)) return r;
  return MD_OK;
}

extern "C" int md_sim_destroy(md_sim* s) {
  if (!s) return MD_OK;
  if (s->exec) cudaGraphExecDestroy(s->exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  md_nlist_destroy(s->nl);
  md_cell_list_destroy(s->cl);
  delete s;
  return MD_OK;
}

extern "C" int md_sim_create(md_sim** out, md_system* sys, md_engine* eng, const md_sim_params* p) {
  if (!out || !sys || !eng || !p || !(p->skin >= 0) || !(p->cell_size > 0)) {
    md_set_error("md_sim_create: bad arguments");
    return MD_ERR_BADARG;
  }
  if (!eng->has_lj) { md_set_error("md_sim_create: register a non-bonded interaction first"); return MD_ERR_BADARG; }
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
  double rlist = rmax + p->skin;
  if ((r = md_nlist_create(&s->nl, sys, rlist, p->skin, p->expansion > 0 ? p->expansion : 1.0, p->nl_mode))) return fail(r);
  if ((r = md_cell_list_rebuild(s->cl, sys))) return fail(r);
  if ((r = md_nlist_fit(s->nl, sys, s->cl))) return fail(r);
  // head room for the run: 25% + 32 over the largest list of the start configuration
  {
    DevState hs;
    if ((r = sys->read_state(hs))) return fail(r);
    int want = ((int)(hs.max_nnb * 1.25) + 32 + 7) & ~7;
    if (want > s->nl->cap) {
      cudaFree(s->nl->list);
      s->nl->list = nullptr;
      s->nl->cap = want;
      if (cudaMalloc(&s->nl->list, sizeof(int) * (size_t)want * sys->N) != cudaSuccess) return fail(md_cuda_fail(cudaGetLastError(), "nlist realloc"));
      if ((r = md_nlist_rebuild(s->nl, sys, s->cl))) return fail(r);
    }
  }
  // initial forces and pressure
  Recorder rec;
  rec.stream = sys->stream;
  if ((r = clear_stats_impl(sys, &rec, MD_STAT_NB_ENERGY, 4))) return fail(r);
  if ((r = lj_apply_impl(eng, sys, s->nl, true, true, &rec))) return fail(r);
  {
    md_langevin_params keep = sys->lv;
    sys->lv.dt = 1e-300;  // kinetic tensor and pressure with no kick
    r = langevin_step2_impl(sys, &rec);
    sys->lv = keep;
    if (r) return fail(r);
  }
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  if (p->use_graph) {
    if (cudaGraphCreate(&s->graph, 0) != cudaSuccess) return fail(md_cuda_fail(cudaGetLastError(), "graph create"));
    Recorder g;
    g.graph = s->graph;
    g.stream = sys->stream;
    if ((r = record_step(s, &g))) return fail(r);
    if (cudaGraphInstantiate(&s->exec, s->graph, 0) != cudaSuccess) return fail(md_cuda_fail(cudaGetLastError(), "graph instantiate"));
  }
  *out = s;
  return MD_OK;
}

extern "C" int md_sim_run(md_sim* s, int nsteps) {
  if (!s || nsteps < 0) return MD_ERR_BADARG;
  md_system* sys = s->sys;
  for (int i = 0; i < nsteps; ++i) {
    if (s->exec) {
      MD_CUDA(cudaGraphLaunch(s->exec, sys->stream));
    } else {
      Recorder rec;
      rec.stream = sys->stream;
      if (int r = record_step(s, &rec)) return r;
    }
  }
  s->steps += nsteps;
  return MD_OK;
}

extern "C" int md_sim_counters(md_sim* s, int64_t* steps, int64_t* rebuilds, int* flags) {
  if (!s) return MD_ERR_BADARG;
  DevState hs;
  if (int r = s->sys->read_state(hs)) return r;
  if (steps) *steps = s->steps;
  if (rebuilds) *rebuilds = (int64_t)hs.rebuilds + ((hs.flags & FLAG_REBUILD) ? 1 : 0);
  if (flags) *flags = (int)hs.flags;
  if (hs.flags & FLAG_NL_OVERFLOW) {
    md_set_error("neighbour list overflow during the run (largest list %d, capacity %d)", hs.max_nnb, s->nl->cap);
    return MD_ERR_NLIST_OVERFLOW;
  }
  if (hs.flags & FLAG_NAN) { md_set_error("non-finite coordinates during the run"); return MD_ERR_BADARG; }
  return MD_OK;
}
