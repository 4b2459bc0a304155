#!/usr/bin/env python3
"""Benchmark: MD steps/s on the 65536-atom liquid-vapour LJ slab.

Workload (one step = one Langevin NPT MD step of the whole slab through the
graph-captured driver): 40 x 40 x 160 sigma box, liquid rho* 0.78 for
|z - 80| < 24.84, vapour 0.02, adaptive per-bin LJ cutoff in [2.5, 5.0]
(AdaptRCut at target 0.02, re-estimated every 2000 steps), skin 0.6,
Langevin NPT with P_zz = 0 (x, y fixed), dt 0.005, T* 0.85, from the
committed start tests/golden/slab65536_start.npz.
`value` is the mixed-precision path (FP32 pair math, FP64 accumulation);
the plain FP64 path runs the same steps and is reported beside it, with the
force RMS error of mixed against FP64 and of both against long-cutoff FP64
forces, beside the AdaptRCut a-priori estimate.

python bench.py --gpus N --steps K --warmup W [--impl reference]
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time
from types import SimpleNamespace

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "md.error_b200"))
sys.path.insert(0, ROOT)

METRIC = "MD steps/s at 64k-atom slab, force RMS err <=1e-4 vs FP64; mixed vs plain FP64"
DT = 0.005
TEMP = 0.85
# Verlet skin of the slab runs: a tuning parameter (the interacting pairs are
# fixed by rc); 0.5-0.7 is the measured optimum on B200 (fewer list builds
# against longer lists).  The LJ-fluid configuration specifies 0.3, which the
# other workloads and the CPU baseline keep.
SKIN = 0.6
SKIN_SPEC = 0.3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--equil", type=int, default=4000,
                    help="untimed relaxation steps of the other workloads' starts (the slab's start is "
                         "committed)")
    ap.add_argument("--workload", default="lj_slab", choices=list(WORKLOADS),
                    help="lj_slab: the 65536-atom slab of the headline metric (default); the others "
                         "time the remaining named systems")
    ap.add_argument("--launch", default="graph", choices=["graph", "direct"],
                    help="direct: launch each step's kernels on the stream instead of one CUDA graph "
                         "(rebuild kernels gated on the device flag); for profilers that do not "
                         "descend into conditional graph nodes")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def replica_rate(torch, steps, t_local, world, device):
    """Whole-job steps/s of `world` independent replicas: every rank ran
    `steps` steps; the job's time is the slowest rank's (max over ranks,
    all-reduced on `device` through the initialised process group)."""
    t_max = t_local
    if world > 1:
        tt = torch.tensor([t_local], device=device, dtype=torch.float64)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        t_max = float(tt.item())
        torch.distributed.barrier()
    return world * steps / t_max, t_max


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(kernel):
    """DRAM bytes (read + write) per launch of `kernel` from its committed ncu
    summary under profiles/, or None when there is none."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_slab65536.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch:"):
                    return float(line.split(":", 1)[1])
    except (OSError, ValueError):
        pass
    return None


START = os.path.join(ROOT, "tests", "golden", "slab65536_start.npz")


def load_slab_start():
    """The committed start of the 65,536-atom slab (tests/golden/make_slab_start.py):
    random sequential addition + 4000 Langevin NVT steps, and the adaptive cutoff
    lattice of the reference's AdaptRCut at target 0.02.  Plain numpy: both arms
    read it, neither generates or relaxes it."""
    z = np.load(START)
    return SimpleNamespace(name="lj_slab", pos=z["pos"].astype(np.float64), vel=z["vel"].astype(np.float64),
                           box=np.asarray(z["box"], np.float64), lattice=np.asarray(z["lattice"], np.float32),
                           n=int(z["pos"].shape[0]), relax=int(z["relax_steps"]))


RC_MIN, RC_MAX, RC_STEP = 2.5, 5.0, 0.5
TARGET_PREC = 0.02      # targetPrec of ENG/app/lj.nhc-xtc.cu:57
SAMPLE_EVERY, UPDATE_EVERY = 40, 2000  # densityProfileSamplingFeq, rcutUpdateFeq (:49-51)
GAMMA_T, TAU_P, KAPPA_T = 1.0, 2.0, 0.1
RC_LONG = 10.0          # cutoff of the long-range FP64 reference forces (+ LFC)


def slab_config(s, world):
    """The workload as both arms state it (identical dicts)."""
    counts = {float(v): int((s.lattice == v).sum()) for v in np.unique(s.lattice)}
    return {"workload": "lj_slab_65536_npt", "n_atoms": s.n, "box": s.box.tolist(),
            "rc": f"adaptive per-bin lattice {tuple(s.lattice.shape)} from the reference AdaptRCut at target "
                  f"{TARGET_PREC}, rc {RC_MIN}..{RC_MAX} step {RC_STEP}, bins per rc {counts}; re-estimated every "
                  f"{UPDATE_EVERY} steps from samples every {SAMPLE_EVERY}",
            "skin": SKIN, "dt": DT, "T": TEMP,
            "ensemble": f"Langevin NPT Pzz=0 (gamma {GAMMA_T}, tau_P {TAU_P}, kappa_T {KAPPA_T})",
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "GPU arm: flushed (256 MB write) between timed steps; CPU arm: no flush",
            "start": f"tests/golden/slab65536_start.npz: random sequential addition (0.8 sigma) + {s.relax} "
                     f"Langevin NVT steps on the CPU oracle"}


def make_sim(mdf, s, prec, lattice, seed=1, use_graph=True, attach_arc=True):
    sys_ = mdf.MDSystem(s.pos, s.box, vel=s.vel, precision=prec)
    mdf.AssignRCut(lattice).assign(sys_)
    eng = mdf.InteractionEngine(sys_)
    eng.registNonBondedInteraction(1.0, 1.0, 0.0)
    lv = mdf.langevin_params(dt=DT, temperature=TEMP, gamma_t=GAMMA_T, tau_p=TAU_P, kappa_t=KAPPA_T,
                             p_ref=(0.0, 0.0, 0.0), npt_dirs=4, seed=seed)
    sim = mdf.Simulation(sys_, eng, skin=SKIN, cell_size=2.8, lv=lv, expansion=1.5, use_graph=use_graph,
                         max_rcut=RC_MAX)
    arc = None
    if attach_arc:
        arc = mdf.AdaptRCutEstimator(sys_, refh=1.0, rcmin=RC_MIN, rcmax=RC_MAX, rcstep=RC_STEP)
        sim.attach_adapt_rcut(arc, sample_every=SAMPLE_EVERY, update_every=UPDATE_EVERY, prec=TARGET_PREC)
    return sys_, eng, sim, arc


def time_steps(torch, sim, stream, steps, flush, nvtx_range=None):
    """Per-step CUDA-event timing; L2 is flushed between timed steps.  The loop
    is wrapped in an NVTX range when one is named, so that a profiler can be
    restricted to the timed launches (ncu --nvtx --nvtx-include <name>/)."""
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    if nvtx_range:
        torch.cuda.nvtx.range_push(nvtx_range)
    with torch.cuda.stream(stream):
        for a, b in ev:
            flush.zero_()
            a.record(stream)
            sim.run(1)
            b.record(stream)
    torch.cuda.synchronize()
    if nvtx_range:
        torch.cuda.nvtx.range_pop()
    return sum(a.elapsed_time(b) for a, b in ev) / 1e3


def fitted_list(mdf, sys_, skin=SKIN, cell=2.8):
    cl = mdf.CellList(sys_, cell)
    cl.rebuild()
    rc = sys_.rcut()
    nl = mdf.NeighborList(sys_, float(rc.max()) + skin, skin, expansion=1.5)
    nl.fit(sys_, cl)
    return cl, nl


def time_kernels(torch, mdf, sys_, eng, stream, reps=50):
    """Average CUDA-event duration of the LJ force kernel on the bench state (a
    list built the way the driver builds it), of one list build, and the list's
    entry count P."""
    cl, nl = fitted_list(mdf, sys_)
    counts, _ = nl.lists()
    P = int(counts.sum())
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the force kernel as the step runs it: statistics left as per-warp rows,
    # which the step's closing kick adds up
    with torch.cuda.stream(stream):
        for _ in range(5):
            eng.applyNonBondedInteraction(sys_, nl, with_stats="rows")
        a.record(stream)
        for _ in range(reps):
            eng.applyNonBondedInteraction(sys_, nl, with_stats="rows")
        b.record(stream)
    torch.cuda.synchronize()
    t_lj = a.elapsed_time(b) / 1e3 / reps
    # list build on the same state (each call: flag clear, build, 1 status read)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(10)]
    with torch.cuda.stream(stream):
        nl.rebuild(sys_, cl)
        for x, y in ev:
            x.record(stream)
            nl.rebuild(sys_, cl)
            y.record(stream)
    torch.cuda.synchronize()
    t_nl = sum(x.elapsed_time(y) for x, y in ev) / 1e3 / len(ev)
    del nl, cl
    # entries within rc_i (the pairs that interact): a list with zero skin
    cl0, nl0 = fitted_list(mdf, sys_, skin=0.0)
    c0, _ = nl0.lists()
    return t_lj, P, t_nl, int(c0.sum())


def start_forces(mdf, s, prec):
    """Forces of the adaptive-cutoff LJ on the start configuration."""
    sys_ = mdf.MDSystem(s.pos, s.box, precision=prec)
    mdf.AssignRCut(s.lattice).assign(sys_)
    _, nl = fitted_list(mdf, sys_)
    eng = mdf.InteractionEngine(sys_)
    eng.registNonBondedInteraction(1.0, 1.0, 0.0)
    eng.clearInteraction()
    eng.applyNonBondedInteraction(sys_, nl, with_stats=True)
    return sys_, sys_.forces()


def long_cutoff_forces(mdf, s):
    """FP64 forces at a uniform cutoff of 10 sigma plus the long-range force
    correction (ForceCorr on 1-sigma bins of this configuration's density, averaged
    over x and y): the
    near-exact LJ forces the adaptive cutoff approximates.  The FP64 kernel that
    computes them is the one the tests pin to the all-pairs oracle."""
    sys_ = mdf.MDSystem(s.pos, s.box, precision=1)
    sys_.set_rcut(np.full(s.n, RC_LONG, np.float32))
    fc = mdf.ForceCorr(sys_, RC_LONG, refh=1.0)
    fc.deposite()
    fc.update()         # DensityProfile::calculate of the one sample
    rho = fc.profile()  # averaged over the slab's homogeneous x and y
    fc.set_profile(np.broadcast_to(rho.mean(axis=(0, 1), keepdims=True), rho.shape))
    fc.update()
    fc.assign()
    _, nl = fitted_list(mdf, sys_, skin=0.0, cell=5.0)
    eng = mdf.InteractionEngine(sys_)
    eng.registNonBondedInteraction(1.0, 1.0, 0.0)
    eng.setForceCorrection(fc)
    eng.clearInteraction()
    eng.applyNonBondedInteraction(sys_, nl, with_stats=True)
    return sys_.forces()


def apriori_error(mdf, sys_, s):
    """RMS over atoms of the AdaptRCut error estimate (ENG/src/AdaptRCut.cu calError)
    of each atom's bin at the cutoff the lattice gives it, for this configuration's
    density: one deposit, averaged over x and y (the slab is homogeneous there;
    a single sample leaves most vapour bins empty)."""
    arc = mdf.AdaptRCutEstimator(sys_, refh=1.0, rcmin=RC_MIN, rcmax=RC_MAX, rcstep=RC_STEP)
    arc.clearData()
    arc.deposite()
    arc.update(TARGET_PREC)  # DensityProfile::calculate of the one sample
    rho = arc.profile()
    arc.set_profile(np.broadcast_to(rho.mean(axis=(0, 1), keepdims=True), rho.shape))
    arc.update(TARGET_PREC)
    err = arc.error()  # (nrc, nx, ny, nz)
    idx = np.rint((s.lattice - RC_MIN) / RC_STEP).astype(np.int64)
    per_bin = np.take_along_axis(err, idx[None], 0)[0]
    n = np.array(arc.n)
    b = np.clip(np.floor(s.pos / s.box * n).astype(np.int64), 0, n - 1)
    e_atom = per_bin[b[:, 0], b[:, 1], b[:, 2]]
    return float(np.sqrt((e_atom ** 2).mean())), float(per_bin.max())


def cpu_port(s, nsteps):
    """The oracle's CPU FP64 Langevin NPT MD (cell + Verlet list, OpenMP) on the
    start, at the GPU arm's skin and lattice."""
    from oracle import oracle as orc
    kw = dict(dt=DT, temperature=TEMP, gamma_t=GAMMA_T, skin=SKIN, lattice=s.lattice, tau_p=TAU_P,
              kappa_t=KAPPA_T, p_ref=(0, 0, 0), npt_dirs=4, seed=1, cap=1024)
    orc.md_langevin_run(s.pos, s.vel, s.box, 1, **kw)  # warm (page in, list build)
    t = time.perf_counter()
    out = orc.md_langevin_run(s.pos, s.vel, s.box, nsteps, **kw)
    el = time.perf_counter() - t
    if out["status"] != 0:
        raise RuntimeError(f"CPU port failed: status {out['status']}")
    return nsteps / el, orc.num_threads()


def reference_loop(pairs_per_step):
    """The reference's own CPU LJ loop (force.kernel/test.kernels/app/explicit.cpp,
    built as shipped into oracle/_ref/ref_explicit_lj): its fixed sample of
    10,000 atoms x 39,999 list entries (4.0e8 pair forces with Newton's third
    law), one copy per host core at once.  Returns the aggregate pair rate and
    the slab steps/s it projects for the force loop alone (pairs_per_step =
    half the list entries of one slab step)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_explicit_lj")
    if not os.access(exe, os.X_OK):
        return None
    cores = os.cpu_count() or 1
    t = time.perf_counter()
    procs = [subprocess.Popen([exe], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
             for _ in range(cores)]
    reals = []
    for p in procs:
        out, _ = p.communicate(timeout=600)
        for ln in out.splitlines():
            if ln.startswith("system:"):
                reals.append(float(ln.split("real:")[1]))
    wall = time.perf_counter() - t
    if len(reals) != cores:
        return None
    pairs = 10000 * 39999
    rate = pairs * cores / max(reals)
    return {"pairs_per_s": rate, "pairs_per_s_per_core": pairs / float(np.median(reals)), "cores": cores,
            "wall_s": wall, "slab_pairs_per_step": pairs_per_step,
            "projected_force_loop_steps_per_s": rate / pairs_per_step,
            "sample": "force.kernel/test.kernels/app/explicit.cpp as shipped (g++ -O3 -msse -msse2): FP32 LJ "
                      "over its own random list of 10,000 x 39,999 entries, Newton's third law, no cutoff "
                      "test or periodic images; one copy per core"}


WORKLOADS = ("lj_slab", "lj_fluid", "charged_fluid", "charged_slab", "charged_lj_slab", "lj_slab_lfc",
             "spme_adjoint")


def run_workload(args):
    """The other named systems, one JSON line each (rank 0): steps/s of the
    mixed path and of plain FP64 through the graph-captured driver, force RMS
    error of mixed against FP64 on the start configuration, per-step device
    time.  lj_fluid: 4000-atom fcc LJ fluid, rc 2.5 shifted, Langevin NVT
    gamma 0.1, dt 0.005.  charged_fluid: 20736 unit charges in a 30^3 box, LJ
    rc 3.0 + real-space Ewald (beta 0.95, rc 3.0) + ik SPME 64^3 order 6,
    Langevin NVT T 1, dt 0.002.  charged_slab: 1048576 unit charges, liquid
    0.8 for |z - 200| < 64 in 100 x 100 x 400, vapour 0.01, SPME 128 x 128 x
    512 order 6, beta for a real-space error of 1e-4 at rc 3.0; adaptive
    per-atom cutoff 3.0..5.0 (AdaptRCut on 2-sigma bins of the density
    sampled during the relaxation, re-estimated on the reference's schedule).
    charged_lj_slab: the LJ+SPME slab, the 65,536-atom slab start
    (tests/golden/slab65536_start.npz) with half +1 and half -1 charges
    (seeded), LJ + real-space Ewald at the per-atom adaptive cutoff 3.0..5.0
    and ik SPME order 6, beta and the mesh chosen as for charged_slab, the
    same relaxation, schedule and sampled error against a converged sum.
    lj_slab_lfc: the 65536-atom slab at a uniform cutoff 3.5 with the
    long-range force correction (ForceCorr on 1-sigma bins: field from the
    density sampled during the relaxation, then assigned every 40 steps,
    sampled every 40 and re-estimated every 2000, the fcorr app's schedule),
    Langevin NVT T 0.85, dt 0.005.
    Charged systems also report the a-priori RMS force errors of the real
    space (errorEstimatePME at rc 3.0) and of the ik-SPME interpolation
    (errorEstimateInterpolRec) beside the measured mixed-vs-FP64 error."""
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    import mdforce as mdf
    w = args.workload
    lfc = w == "lj_slab_lfc"
    if w == "lj_fluid":
        s = mdf.systems.lj_fluid_fcc()
        rc, dt, T, gamma, coul = 2.5, 0.005, 1.0, 0.1, None
        shift = -4.0 * (rc ** -12 - rc ** -6)
    elif lfc:
        s = mdf.systems.lj_slab()
        rc, dt, T, gamma, shift, coul = 3.5, DT, TEMP, 1.0, 0.0, None
    elif w == "charged_fluid":
        s = mdf.systems.charged_fluid()
        rc, dt, T, gamma, shift = 3.0, 0.002, 1.0, 1.0, 0.0
        coul = dict(beta=0.95, K=(64, 64, 64), order=6)
    elif w == "charged_lj_slab":
        st = load_slab_start()
        s = SimpleNamespace(name=w, n=st.n, pos=st.pos, vel=st.vel, box=st.box,
                            charge=mdf.systems.charges(st.n, 7))
        rc, dt, T, gamma, shift = 3.0, 0.002, 1.0, 1.0, 0.0
        coul = dict(beta=None, K=(64, 64, 256), order=6)
    else:
        s = mdf.systems.charged_slab()
        rc, dt, T, gamma, shift = 3.0, 0.002, 1.0, 1.0, 0.0
        coul = dict(beta=None, K=(128, 128, 512), order=6)
    adaptive = w in ("charged_slab", "charged_lj_slab")
    arc_kw = dict(refh=2.0, rcmin=3.0, rcmax=5.0, rcstep=0.5)
    lattice = [None]
    lfc_profile = [None]
    keep = []

    def build(prec, pos, vel, attach=True):
        sys_ = mdf.MDSystem(pos, s.box, vel=vel, charge=s.charge, precision=prec)
        if lattice[0] is None:
            sys_.set_rcut(np.full(s.n, rc, np.float32))
        else:
            mdf.AssignRCut(lattice[0]).assign(sys_)
        eng = mdf.InteractionEngine(sys_)
        eng.registNonBondedInteraction(1.0, 1.0, shift)
        sp = None
        if coul is not None:
            beta = coul["beta"] or mdf.choose_beta(sys_, rc, 1e-4)
            coul["beta"] = beta
            mdf.registCoulomb(eng, beta)
            sp = mdf.SPME(sys_, coul["K"], coul["order"], beta, "ik")
        lv = mdf.langevin_params(dt=dt, temperature=T, gamma_t=gamma, seed=1 + rank)
        sim = mdf.Simulation(sys_, eng, skin=SKIN_SPEC, cell_size=rc + SKIN_SPEC, lv=lv, expansion=1.5, spme=sp,
                             use_graph=args.launch == "graph", max_rcut=arc_kw["rcmax"] if adaptive else 0.0)
        if adaptive and attach and lattice[0] is not None:
            arc = mdf.AdaptRCutEstimator(sys_, **arc_kw)
            sim.attach_adapt_rcut(arc, sample_every=SAMPLE_EVERY, update_every=UPDATE_EVERY, prec=TARGET_PREC)
        if lfc and lfc_profile[0] is not None:
            fc = mdf.ForceCorr(sys_, rc, refh=1.0)
            fc.set_profile(lfc_profile[0])
            fc.update()
            fc.assign()
            if attach:
                sim.attach_force_corr(fc, assign_every=40, sample_every=SAMPLE_EVERY, update_every=UPDATE_EVERY)
            else:
                eng.setForceCorrection(fc)
            keep.append(fc)
        return sys_, eng, sim

    stream = torch.cuda.Stream()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    vel = s.vel if s.vel is not None else mdf.systems.maxwell(s.n, T, 11)
    # relaxation of the start (random sequential addition / lattice), not timed
    sys0, _, sim0 = build(0, s.pos, vel)
    n_equil = args.equil if args.equil != 4000 else 1000
    if adaptive:
        # density sampled over the second half of the relaxation -> cutoff lattice
        arc0 = mdf.AdaptRCutEstimator(sys0, **arc_kw)
        done = 0
        while done < max(n_equil, SAMPLE_EVERY):
            sim0.run(SAMPLE_EVERY)
            done += SAMPLE_EVERY
            if done > n_equil // 2:
                arc0.deposite()
        arc0.update(TARGET_PREC)
        rcl, _, _ = arc0.rcut()
        lattice[0] = rcl.astype(np.float32)
        rc_info = (f"adaptive per-bin lattice {arc0.n} from AdaptRCut at target {TARGET_PREC}, rc 3.0..5.0 step "
                   f"0.5 (2-sigma bins); bins per rc {({float(v): int((rcl == v).sum()) for v in np.unique(rcl)})}")
        del arc0
    elif lfc:
        fc0 = mdf.ForceCorr(sys0, rc, refh=1.0)
        done = 0
        while done < max(n_equil, SAMPLE_EVERY):
            sim0.run(SAMPLE_EVERY)
            done += SAMPLE_EVERY
            if done > n_equil // 2:
                fc0.deposite()
        fc0.update()
        lfc_profile[0] = fc0.profile()
        rc_info = f"uniform {rc} with the long-range force correction (bins {fc0.n})"
        del fc0
    else:
        sim0.run(n_equil)
        rc_info = rc
    pos, vel = sys0.positions(), sys0.velocities()
    del sim0, sys0
    chosen = None
    if adaptive:
        # beta and the mesh from the error estimates of the relaxed charge profile
        # (md_choose_spme_params) at a total target of 1e-4; the configuration's
        # own mesh is reported beside it with its estimate at the chosen beta
        sysc = mdf.MDSystem(pos, s.box, charge=s.charge, precision=1)
        config_mesh = coul["K"]
        # the smallest total target the estimates can meet with order 6 within
        # the mesh limits (1e-4 first)
        for target in (1e-4, 2e-4, 5e-4, 1e-3, 2e-3):
            try:
                beta, K, e_dir, e_rec = mdf.choose_spme_params(sysc, rc, coul["order"], target, kmax=1024)
                break
            except mdf.MDExcptBadArgument:
                continue
        else:
            raise RuntimeError("no SPME parameters meet 2e-3 within the mesh limits")
        e_cfg = mdf.ErrorEstimate_SPME_Ik(config_mesh, s.box, beta, coul["order"])
        e_cfg.deposit(sysc)
        cfg_max = float(np.nanmax(e_cfg.rms(1.0)))
        del e_cfg, sysc
        coul["beta"], coul["K"] = beta, K
        chosen = {"target": target, "target_asked": 1e-4, "beta": beta, "mesh": list(K), "real_space_max_bin": e_dir,
                  "spme_ik_max_bin": e_rec, "total_max_bin": float(np.hypot(e_dir, e_rec)),
                  "config_mesh": list(config_mesh), "config_mesh_spme_ik_max_bin": cfg_max}
    out = {}
    for prec in (0, 1):
        sys_, eng, sim = build(prec, pos, vel)
        sys_.set_stream(stream.cuda_stream)
        sim.run(args.warmup)
        t = time_steps(torch, sim, stream, args.steps, flush, nvtx_range="timed" if prec == 0 else None)
        out[prec] = (args.steps / t, sys_, sim)
    # force RMS error of mixed against FP64 on the relaxed configuration
    F = {}
    apriori = None
    for prec in (0, 1):
        sys_, _, sim = build(prec, pos, vel, attach=False)
        F[prec] = sys_.forces()
        if coul is not None and prec == 1:
            e_dir, _ = mdf.errorEstimatePME(sys_, coul["K"], coul["beta"], rc)
            e_rec = mdf.errorEstimateInterpolRec(sys_, coul["K"], coul["order"], coul["beta"])
            apriori = {"real_space_rc3": e_dir, "spme_ik_interpolation": e_rec}
    d = F[0] - F[1]
    err_abs = float(np.sqrt((d ** 2).sum(1).mean()))
    err_rel = float(np.sqrt((d ** 2).sum() / (F[1] ** 2).sum()))
    sampled = None
    if chosen is not None:
        sampled = sampled_electrostatics_error(mdf, s, pos, lattice[0], arc_kw, coul)
    if rank == 0:
        line = {"metric": "MD steps/s", "value": out[0][0], "unit": "steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / out[0][0],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 pair math / f64 accumulation", "data": "synthetic",
                "config": {"workload": w, "n_atoms": s.n, "box": s.box.tolist(), "rc": rc_info, "skin": SKIN_SPEC,
                           "dt": dt, "T": T, "ensemble": "Langevin NVT",
                           "electrostatics": None if coul is None else
                           dict(beta=coul["beta"], mesh=list(coul["K"]), order=coul["order"], method="ik"),
                           "l2": "flushed (256 MB write) between timed steps"},
                "fp64_steps_per_s": out[1][0], "speedup_vs_fp64": out[0][0] / out[1][0],
                "force_rms_err_vs_fp64": {"abs": err_abs, "rel": err_rel},
                "tau_per_day": out[0][0] * dt * 86400}
        if apriori is not None:
            line["apriori_force_rms_error"] = apriori
        if chosen is not None:
            line["electrostatics_choice"] = chosen
            line["force_rms_err_vs_converged"] = sampled
        print(json.dumps(line), flush=True)
    return 0


def sampled_electrostatics_error(mdf, s, pos, lattice, arc_kw, coul, nsample=4096, seed=3):
    """Electrostatic forces of the run's parameters (real-space Ewald at the
    per-atom adaptive cutoffs >= 3.0, ik SPME at the chosen beta, mesh, order 6)
    in both precisions against a converged FP64 Ewald sum, on nsample atoms
    drawn without replacement: real space at a uniform 7.0 (erfc(7 beta) below
    1e-20) and SPME on twice the mesh per axis (at most 1024) with B-spline
    order 12 (its homogeneous a-priori estimate is reported).  Only the
    electrostatics enter (LJ switched off)."""
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(s.n, size=min(nsample, s.n), replace=False))
    beta = coul["beta"]

    def forces(prec, rc_uniform, K, order):
        sys_ = mdf.MDSystem(pos, s.box, charge=s.charge, precision=prec)
        if rc_uniform is None:
            mdf.AssignRCut(lattice).assign(sys_)
        else:
            sys_.set_rcut(np.full(s.n, rc_uniform, np.float32))
        rmax = float(sys_.rcut().max())
        eng = mdf.InteractionEngine(sys_)
        eng.registNonBondedInteraction(0.0, 1.0, 0.0)
        mdf.registCoulomb(eng, beta)
        cl = mdf.CellList(sys_, max(3.3, rmax / 2))
        cl.rebuild()
        nl = mdf.NeighborList(sys_, rmax + 0.3, 0.3, expansion=1.3)
        nl.fit(sys_, cl)
        eng.clearInteraction()
        eng.applyNonBondedInteraction(sys_, nl)
        mdf.SPME(sys_, K, order, beta, "ik").apply()
        est = mdf.errorEstimateInterpolRec(sys_, K, order, beta) if prec == 1 else None
        return sys_.forces()[idx], est

    fine = tuple(min(1024, 2 * k) for k in coul["K"])
    Fref, est_ref = forces(1, 7.0, fine, 12)
    out = {"sample": f"{len(idx)} atoms", "reference": {"real_space_rc": 7.0, "mesh": list(fine), "order": 12,
                                                          "spme_ik_apriori": est_ref}}
    for prec, name in ((0, "mixed"), (1, "fp64")):
        F, _ = forces(prec, None, coul["K"], coul["order"])
        d = F - Fref
        out[name] = float(np.sqrt((d ** 2).sum(1).mean()))
    return out


def run_spme_adjoint(args):
    """The SPME adjoint on a batch of interpolation bases: 20736 unit charges
    (the charged fluid), mesh 64^3, beta 0.95, the Hermite basis of the
    B-spline of order 4 and of order 6 (support CC = order/2, 16 bins: 32
    coefficients) plus N(0, 0.1) perturbations, 8 candidates per call.  One
    step is one call of the energy with dE/dq, dE/dr, dE/dc and one of the
    force-error functional (against the unperturbed basis's forces) with
    dL/dq, dL/dr, dL/dc for all 8 candidates, FP64.  value: candidates per
    second at order 6 (device time, inputs resident, L2 flushed between
    steps); e2e: the same through pinned host arrays copied in and every
    gradient copied out inside the timed region."""
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    import mdforce as mdf
    s = mdf.systems.charged_fluid()
    dev = torch.device("cuda", local)
    K, beta, nbin, ncand = (64, 64, 64), 0.95, 16, 8
    rng = np.random.default_rng(7)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    per_order = {}
    for order in (4, 6):
        CC = order / 2.0
        hs = mdf.optibasis.HermiteSPME(s.n, K, s.box, beta, CC, nbin)
        base = mdf.optibasis.bspline_initial_basis(CC, nbin, order)
        cand = base[None, :] + rng.normal(0.0, 0.1, size=(ncand, base.size))
        q = torch.tensor(s.charge, dtype=torch.float64, device=dev)
        r = torch.tensor(s.pos, dtype=torch.float64, device=dev)
        c = torch.tensor(cand, dtype=torch.float64, device=dev)
        fref = hs.energy(q, r, torch.tensor(base, dtype=torch.float64, device=dev), forces=True)["forces"][0].clone()

        def step():
            a = hs.energy(q, r, c, grads=True)
            b = hs.force_error(q, r, c, fref, grads=True)
            return a, b

        for _ in range(max(args.warmup, 3)):
            step()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for x, y in ev:
            flush.fill_(1)
            x.record(stream)
            step()
            y.record(stream)
        torch.cuda.synchronize()
        t_dev = sum(x.elapsed_time(y) for x, y in ev) / 1e3 / len(ev)
        # end to end: host inputs in, gradients out, every step
        hq = torch.tensor(s.charge, dtype=torch.float64).pin_memory()
        hr = torch.tensor(s.pos, dtype=torch.float64).pin_memory()
        hc = torch.tensor(cand, dtype=torch.float64).pin_memory()
        hf = fref.cpu().pin_memory()
        outs = {k: torch.empty(sh, dtype=torch.float64).pin_memory() for k, sh in
                (("e", (ncand,)), ("gq", (ncand, s.n)), ("gr", (ncand, s.n, 3)), ("gc", (ncand, hs.ncoef)),
                 ("l", (ncand,)), ("lq", (ncand, s.n)), ("lr", (ncand, s.n, 3)), ("lc", (ncand, hs.ncoef)))}
        h2d = sum(t.numel() * 8 for t in (hq, hr, hc, hf))
        d2h = sum(t.numel() * 8 for t in outs.values())
        torch.cuda.synchronize()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(args.steps):
            dq, dr, dc, df = (hq.to(dev, non_blocking=True), hr.to(dev, non_blocking=True),
                              hc.to(dev, non_blocking=True), hf.to(dev, non_blocking=True))
            A = hs.energy(dq, dr, dc, grads=True)
            Bv = hs.force_error(dq, dr, dc, df, grads=True)
            for k, v in (("e", A["energy"]), ("gq", A["dE_dq"]), ("gr", A["dE_dr"]), ("gc", A["dE_dc"]),
                         ("l", Bv["loss"]), ("lq", Bv["dL_dq"]), ("lr", Bv["dL_dr"]), ("lc", Bv["dL_dc"])):
                outs[k].copy_(v, non_blocking=True)
        a1.record(stream)
        torch.cuda.synchronize()
        t_e2e = a0.elapsed_time(a1) / 1e3 / args.steps
        per_order[order] = {"device_ms_per_step": t_dev * 1e3, "candidates_per_s": ncand / t_dev,
                            "e2e_candidates_per_s": ncand / t_e2e, "h2d_bytes_per_step": h2d,
                            "d2h_bytes_per_step": d2h, "ncoef": hs.ncoef}
        del hs
    if rank == 0:
        o6 = per_order[6]
        line = {"metric": "SPME adjoint candidate evaluations/s (energy and force-error gradients in q, r, basis)",
                "value": o6["candidates_per_s"], "unit": "candidates/s", "n_gpus": world, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": o6["device_ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "spme_adjoint", "n_atoms": s.n, "box": s.box.tolist(), "mesh": list(K),
                           "beta": beta, "basis": f"Hermite, {nbin} bins, B-spline order 4 and 6 + N(0, 0.1)",
                           "candidates_per_call": ncand, "l2": "flushed (256 MB write) between timed steps"},
                "e2e": {"value": o6["e2e_candidates_per_s"], "unit": "candidates/s",
                        "h2d_bytes_per_step": o6["h2d_bytes_per_step"], "d2h_bytes_per_step": o6["d2h_bytes_per_step"]},
                "per_order": per_order}
        print(json.dumps(line), flush=True)
    return 0


def run_reference(args):
    """The reference arm: the same workload, config, metric and unit on the host
    cores, without the GPU engine (libmdforce is never loaded).  The reference's
    MD engine is CUDA that does not build with nvcc 12.9, so the full step is
    timed on the oracle's CPU port (FP64 Langevin NPT with cell and Verlet lists,
    OpenMP on all host threads) from the committed start, at the GPU arm's skin
    and cutoff lattice; beside it, the reference's own CPU LJ loop
    (explicit.cpp, built as shipped)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    s = load_slab_start()
    # bounded sample: the warm-up steps untimed, then --steps steps (at most ~60 s)
    sps0, cores = cpu_port(s, max(2, min(args.warmup, 5)))
    nsteps = max(2, min(args.steps, int(60 * sps0)))
    sps, cores = cpu_port(s, nsteps)
    half_pairs = None
    try:
        from oracle import oracle as orc
        # list entries of the slab's start at rc_i + skin (the force loop's workload)
        rc = orc.assign_rcut_f32(s.pos, s.box, s.lattice)
        cnt, _ = orc.nlist_allpair_f32(s.pos.astype(np.float32), rc, SKIN, s.box.astype(np.float32))
        half_pairs = int(cnt.sum()) // 2
    except Exception:  # the projection is optional context
        half_pairs = None
    loop = reference_loop(half_pairs) if half_pairs else None
    line = {
        "impl": "reference", "metric": METRIC, "value": sps, "unit": "steps/s", "n_gpus": args.gpus,
        "steps": nsteps, "warmup": args.warmup, "ms_per_step": 1e3 / sps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": slab_config(s, world),
        "cpu_baseline": {"value": sps, "unit": "steps/s", "cores": cores, "kind": "port",
                         "sample": f"{nsteps} Langevin NPT steps of the full 65536-atom slab from the committed "
                                   f"start (oracle CPU FP64 cell + Verlet list LJ, OpenMP, skin {SKIN})"},
        "reference_loop": loop,
        "e2e": {"value": sps, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "spme_adjoint":
        return run_spme_adjoint(args)
    if args.workload != "lj_slab":
        return run_workload(args)
    rank, world, local = dist_env()
    import torch
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    import mdforce as mdf

    s = load_slab_start()
    lattice = s.lattice
    N = s.n
    stream = torch.cuda.Stream()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    # ---- mixed precision path (the headline value)
    use_graph = args.launch == "graph"
    sys_m, eng_m, sim_m, arc_m = make_sim(mdf, s, 0, lattice, seed=1 + rank, use_graph=use_graph)
    sys_m.set_stream(stream.cuda_stream)
    sim_m.run(args.warmup)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    steps0, rebuilds0, _ = sim_m.counters()
    with Clocks(local) as clk:
        t_mixed = time_steps(torch, sim_m, stream, args.steps, flush, nvtx_range="timed")
    steps_done, rebuilds, flags = sim_m.counters()
    rebuild_kind = sim_m.rebuild_kind()
    rebuilds_timed = rebuilds - rebuilds0
    value, t_max = replica_rate(torch, args.steps, t_mixed, world, "cuda")

    # ---- the reference's whole schedule (lj.nhc-xtc.cu:226-254): one 2000-step
    # period with 50 density deposits and one AdaptRCut update + assign + tail
    # pressure correction (host-scheduled between graph launches), warm L2
    torch.cuda.synchronize()
    period = UPDATE_EVERY - (steps_done % UPDATE_EVERY)  # up to and including the next update
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        a.record(stream)
        sim_m.run(period)
        b.record(stream)
    torch.cuda.synchronize()
    t_period = time.perf_counter() - t0
    period_dev = a.elapsed_time(b) / 1e3
    # the density deposit alone, then one update cycle (estimate + assign +
    # pressure correction) on the run's state (the period's update cleared the
    # samples, so the deposits come first)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(10):
        arc_m.deposite()
    sys_m.synchronize()
    deposit_s = (time.perf_counter() - t0) / 10
    t0 = time.perf_counter()
    arc_m.update(TARGET_PREC)
    arc_m.assign()
    arc_m.pressure_correction()
    sys_m.synchronize()
    arc_update_s = time.perf_counter() - t0

    # ---- FP64 path, same steps
    fp64_sps = None
    t_lj64 = None
    if not args.no_fp64:
        sys_d, eng_d, sim_d, _ = make_sim(mdf, s, 1, lattice, seed=1 + rank, use_graph=use_graph)
        sys_d.set_stream(stream.cuda_stream)
        sim_d.run(args.warmup)
        t64 = time_steps(torch, sim_d, stream, args.steps, flush)
        fp64_sps = args.steps / t64
        t_lj64, _, t_nl64, _ = time_kernels(torch, mdf, sys_d, eng_d, stream)
        del sim_d, eng_d, sys_d

    # ---- dominant kernel: LJ forces, algorithmic bytes / CUDA-event duration
    t_lj, P, t_nl, P_rc = time_kernels(torch, mdf, sys_m, eng_m, stream)
    alg_bytes = N * 16 + N * 4 + P * 4 + N * 24  # positions, rcut, list indices, FP64 forces
    alg_bytes_rc = N * 16 + N * 4 + P_rc * 4 + N * 24  # the same with the interacting pairs only
    peak, peak_kind = measured_peak_hbm()
    achieved = alg_bytes / t_lj / 1e9

    # ---- accuracy on the start configuration
    sm, Fm = start_forces(mdf, s, 0)
    _, Fd = start_forces(mdf, s, 1)
    d = Fm - Fd
    rms_abs = float(np.sqrt((d ** 2).sum(1).mean()))
    rms_rel = float(np.sqrt((d ** 2).sum() / (Fd ** 2).sum()))
    Fl = long_cutoff_forces(mdf, s)
    d = Fm - Fl
    err_long = float(np.sqrt((d ** 2).sum(1).mean()))
    d = Fd - Fl
    err_long64 = float(np.sqrt((d ** 2).sum(1).mean()))
    est_rms, est_max = apriori_error(mdf, sm, s)
    del sm

    # ---- end to end through the C ABI with host buffers: one full AdaptRCut
    # period from pinned host arrays, every step's statistics written by the
    # device into its own pinned host row, positions and forces read back
    e2e_steps = max(args.steps, UPDATE_EVERY)
    pin_pos = torch.from_numpy(np.ascontiguousarray(s.pos)).pin_memory()
    pin_vel = torch.from_numpy(np.ascontiguousarray(s.vel)).pin_memory()
    stat_rows = torch.zeros((e2e_steps, mdf.STAT_COUNT), dtype=torch.float64).pin_memory().numpy()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sys_e = mdf.MDSystem(pin_pos.numpy(), s.box, vel=pin_vel.numpy(), precision=0)
    mdf.AssignRCut(lattice).assign(sys_e)
    eng_e = mdf.InteractionEngine(sys_e)
    eng_e.registNonBondedInteraction(1.0, 1.0, 0.0)
    lv = mdf.langevin_params(dt=DT, temperature=TEMP, gamma_t=GAMMA_T, tau_p=TAU_P, kappa_t=KAPPA_T,
                             p_ref=(0.0, 0.0, 0.0), npt_dirs=4, seed=1)
    sim_e = mdf.Simulation(sys_e, eng_e, skin=SKIN, cell_size=2.8, lv=lv, expansion=1.5, max_rcut=RC_MAX)
    arc_e = mdf.AdaptRCutEstimator(sys_e, refh=1.0, rcmin=RC_MIN, rcmax=RC_MAX, rcstep=RC_STEP)
    sim_e.attach_adapt_rcut(arc_e, sample_every=SAMPLE_EVERY, update_every=UPDATE_EVERY, prec=TARGET_PREC)
    sim_e.set_stats_ring(stat_rows)
    t_setup = time.perf_counter() - t0
    t1 = time.perf_counter()
    sim_e.run(e2e_steps)
    sys_e.synchronize()
    fin_pos = sys_e.positions()
    fin_f = sys_e.forces()
    t_run = time.perf_counter() - t1
    e2e_sps = e2e_steps / (t_setup + t_run)
    h2d = (pin_pos.numel() + pin_vel.numel()) * 8 / e2e_steps
    d2h = mdf.STAT_COUNT * 8 + (fin_pos.size + fin_f.size) * 8 / e2e_steps
    # the last row is the last step's statistics; the AdaptRCut update after that
    # step has since replaced the tail pressure correction slots
    keep = [k for k in range(mdf.STAT_COUNT)
            if k not in (mdf.STAT_PRESSURE_CORR_XX, mdf.STAT_PRESSURE_CORR_XX + 1, mdf.STAT_PRESSURE_CORR_XX + 2)]
    if not np.isfinite(stat_rows).all() or not np.array_equal(stat_rows[-1][keep], sys_e.stats()[keep]):
        raise RuntimeError("per-step statistics of the end-to-end run are missing or non-finite")
    del sim_e, arc_e, eng_e, sys_e

    # the first half (with the rebuild folded in, when fused), LJ and the
    # closing kick every step; with the kernel chain instead, bin, scan,
    # scatter, order, gather, copy back, z order and list build per rebuild
    # (every step in direct launch, gated); the density deposit every 40 steps
    # and 3 + 3*3 DFT passes + 7 element-wise kernels per cutoff update (every
    # 2000 steps)
    first, last = steps0, steps0 + args.steps
    n_updates = last // UPDATE_EVERY - first // UPDATE_EVERY
    n_deposits = last // SAMPLE_EVERY - first // SAMPLE_EVERY
    if rebuild_kind == "fused":
        rebuild_launches = 0
    else:
        rebuild_launches = 8 * (rebuilds_timed if rebuild_kind == "conditional" else args.steps)
    launches = 3 * args.steps + rebuild_launches + n_deposits + 22 * n_updates
    cpu = loop = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        n_cpu = 30
        sps_cpu, cores = cpu_port(s, n_cpu)
        cpu = {"value": sps_cpu, "unit": "steps/s", "cores": cores, "kind": "port",
               "sample": f"{n_cpu} Langevin NPT steps of the full 65536-atom slab from the committed start "
                         f"(oracle CPU FP64 cell + Verlet list LJ, OpenMP, skin {SKIN})"}
        loop = reference_loop(P // 2)
    if rank == 0:
        per_step = 1.0 / (value / world)
        amortised = 1.0 / (per_step + (arc_update_s + (UPDATE_EVERY // SAMPLE_EVERY) * deposit_s) / UPDATE_EVERY)
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 pair math / f64 accumulation",
            "data": "synthetic",
            "config": slab_config(s, world),
            "fp64_steps_per_s": fp64_sps,
            "speedup_vs_fp64": (value / world / fp64_sps) if fp64_sps else None,
            "force_rms_err_vs_fp64": {"abs": rms_abs, "rel": rms_rel,
                                      "what": "mixed against the FP64 path, same cutoffs, on the start"},
            "force_rms_err_vs_long_cutoff": {
                "mixed": err_long, "fp64": err_long64,
                "apriori_estimate_rms": est_rms, "apriori_estimate_max_bin": est_max,
                "target": TARGET_PREC,
                "what": f"RMS over atoms of |F - F_ref| (eps/sigma) on the start, F_ref = FP64 forces at a "
                        f"uniform cutoff {RC_LONG} plus the long-range force correction; the estimate is the "
                        f"AdaptRCut error of each atom's bin at its assigned cutoff"},
            "list_rebuilds": rebuilds, "rebuild_kind": rebuild_kind, "tau_per_day": value / world * DT * 86400,
            "schedule": {"period_steps": period, "period_device_s": period_dev, "period_wall_s": t_period,
                         "period_steps_per_s": period / t_period,
                         "arc_update_ms": 1e3 * arc_update_s, "deposit_ms": 1e3 * deposit_s,
                         "steps_per_s_with_arc": amortised,
                         "what": "one AdaptRCut period of the reference app (50 deposits, 1 update + assign + "
                                 "pressure correction per 2000 steps); period_* measured warm-L2 through "
                                 "Simulation.run, steps_per_s_with_arc = flushed value with the measured "
                                 "update and deposit costs amortised"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profiled_traffic("k_lj_mixed"),
                         "kernel": "k_lj_mixed",
                         "kernel_us": t_lj * 1e6, "alg_bytes": alg_bytes, "list_entries": P,
                         "pairs_within_rc": P_rc, "alg_bytes_within_rc": alg_bytes_rc,
                         "frac_within_rc": alg_bytes_rc / t_lj / 1e9 / peak,
                         "peak_kind": peak_kind},
            "kernel_us": {"lj_mixed": t_lj * 1e6, "lj_fp64": None if t_lj64 is None else t_lj64 * 1e6,
                          "nlist_build_mixed": t_nl * 1e6,
                          "nlist_build_fp64": None if t_lj64 is None else t_nl64 * 1e6},
            "e2e": {"value": e2e_sps, "unit": "steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps, "setup_s": t_setup, "run_s": t_run,
                    "steady_steps_per_s": e2e_steps / t_run,
                    "path": "MDSystem from pinned host arrays, AdaptRCut attached on the reference schedule, "
                            "Simulation.run(steps) with every step's statistics written by the device into its "
                            "own pinned host row, positions and forces read back at the end"},
            "gpu_launches": launches,
            "list_rebuilds_timed": rebuilds_timed,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "reference_loop": loop,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
