#!/usr/bin/env python3
"""Benchmark: MD steps/s on the 65536-atom liquid-vapour LJ slab.

Workload (one step = one Langevin NPT MD step of the whole slab through the
graph-captured driver): 40 x 40 x 160 sigma box, liquid rho* 0.78 for
|z - 80| < 24.84, vapour 0.02, adaptive per-slab LJ cutoff in [2.5, 5.0],
skin 0.3, Langevin NPT with P_zz = 0 (x, y fixed), dt 0.005, T* 0.85.
`value` is the mixed-precision path (FP32 pair math, FP64 accumulation);
the plain FP64 path runs the same steps and is reported beside it together
with the force RMS error of mixed against FP64 on the same configuration.

python bench.py --gpus N --steps K --warmup W [--impl reference]
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

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
                    help="untimed NVT relaxation steps of the random start")
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


def build_slab(mdf):
    s = mdf.systems.lj_slab()
    return s


RC_MIN, RC_MAX, RC_STEP = 2.5, 5.0, 0.5
TARGET_PREC = 0.02      # targetPrec of ENG/app/lj.nhc-xtc.cu:57
SAMPLE_EVERY, UPDATE_EVERY = 40, 2000  # densityProfileSamplingFeq, rcutUpdateFeq (:49-51)


def make_sim(mdf, s, prec, lattice, seed=1, npt=True, gamma=1.0, adaptive=True, use_graph=True):
    sys_ = mdf.MDSystem(s.pos, s.box, vel=s.vel, precision=prec)
    if lattice is None:
        sys_.set_rcut(np.full(s.n, RC_MIN, np.float32))
    else:
        mdf.AssignRCut(lattice).assign(sys_)
    eng = mdf.InteractionEngine(sys_)
    eng.registNonBondedInteraction(1.0, 1.0, 0.0)
    lv = mdf.langevin_params(dt=DT, temperature=TEMP, gamma_t=gamma, tau_p=2.0 if npt else 0.0,
                             kappa_t=0.1 if npt else 0.0, p_ref=(0.0, 0.0, 0.0),
                             npt_dirs=4 if npt else 0, seed=seed)
    sim = mdf.Simulation(sys_, eng, skin=SKIN, cell_size=2.8, lv=lv, expansion=1.5, use_graph=use_graph,
                         max_rcut=RC_MAX)
    if adaptive:
        arc = mdf.AdaptRCutEstimator(sys_, refh=1.0, rcmin=RC_MIN, rcmax=RC_MAX, rcstep=RC_STEP)
        sim.attach_adapt_rcut(arc, sample_every=SAMPLE_EVERY, update_every=UPDATE_EVERY, prec=TARGET_PREC)
    return sys_, eng, sim


def equilibrate(mdf, s, nsteps):
    """Relax the random-sequential-addition start (0.8 sigma contacts) by
    Langevin NVT at T*, sampling the density profile every 40 steps; at the end
    the adaptive-cutoff estimate (AdaptRCut, target 0.02, rc 2.5..5.0) of the
    sampled profile gives the per-bin cutoff lattice.  Not timed."""
    sys_, eng, sim = make_sim(mdf, s, 0, None, seed=12345, npt=False, gamma=2.0, adaptive=False)
    arc = mdf.AdaptRCutEstimator(sys_, refh=1.0, rcmin=RC_MIN, rcmax=RC_MAX, rcstep=RC_STEP)
    done = 0
    while done < max(nsteps, SAMPLE_EVERY):
        sim.run(SAMPLE_EVERY)
        done += SAMPLE_EVERY
        if done > nsteps // 2:
            arc.deposite()
    arc.update(TARGET_PREC)
    rc, idx, err = arc.rcut()
    lattice = rc.astype(np.float32)
    sys_.synchronize()
    out = mdf.systems.SyntheticSystem(s.name, sys_.positions(), sys_.box(), sys_.velocities(),
                                      s.charge, dict(s.meta, equilibrated_steps=done))
    counts = {float(v): int((rc == v).sum()) for v in np.unique(rc)}
    info = (f"adaptive per-bin lattice {arc.n} from AdaptRCut at target {TARGET_PREC}, "
            f"rc {RC_MIN}..{RC_MAX} step {RC_STEP}; bins per rc {counts}; "
            f"re-estimated every {UPDATE_EVERY} steps from samples every {SAMPLE_EVERY}")
    del sim, eng, sys_, arc
    return out, lattice, info


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


def time_lj_kernel(torch, mdf, sys_, eng, sim, stream, reps=50):
    """Average duration of the dominant kernel (LJ forces) on the bench state."""
    # the simulation owns its list; time the kernel on a list built the same way
    cl = mdf.CellList(sys_, 2.8)
    cl.rebuild()
    rc = sys_.rcut()
    nl = mdf.NeighborList(sys_, float(rc.max()) + SKIN, SKIN, expansion=1.5)
    nl.fit(sys_, cl)
    counts, _ = nl.lists()
    P = int(counts.sum())
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        for _ in range(5):
            eng.applyNonBondedInteraction(sys_, nl, with_stats=True)
        a.record(stream)
        for _ in range(reps):
            eng.applyNonBondedInteraction(sys_, nl, with_stats=True)
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
    return t_lj, P, t_nl


def force_error(mdf, s, lattice):
    """RMS force error of mixed against FP64 on the same configuration."""
    out = {}
    for prec in (0, 1):
        sys_ = mdf.MDSystem(s.pos, s.box, precision=prec)
        if lattice is None:
            sys_.set_rcut(np.full(s.n, 2.5, np.float32))
        else:
            mdf.AssignRCut(lattice).assign(sys_)
        cl = mdf.CellList(sys_, 2.8)
        cl.rebuild()
        nl = mdf.NeighborList(sys_, float(sys_.rcut().max()) + SKIN, SKIN, expansion=1.5)
        nl.fit(sys_, cl)
        eng = mdf.InteractionEngine(sys_)
        eng.registNonBondedInteraction(1.0, 1.0, 0.0)
        eng.clearInteraction()
        eng.applyNonBondedInteraction(sys_, nl, with_stats=True)
        out[prec] = sys_.forces()
    d = out[0] - out[1]
    rms_abs = float(np.sqrt((d ** 2).sum(1).mean()))
    rms_rel = float(np.sqrt((d ** 2).sum() / (out[1] ** 2).sum()))
    return rms_abs, rms_rel


def cpu_baseline(s, lattice, nsteps):
    from oracle import oracle as orc
    rc = None if lattice is not None else np.full(s.n, 2.5, np.float32)
    kw = dict(dt=DT, temperature=TEMP, gamma_t=1.0, skin=SKIN_SPEC, rcut=rc, lattice=lattice, tau_p=2.0,
              kappa_t=0.1, p_ref=(0, 0, 0), npt_dirs=4, seed=1, cap=1024)
    orc.md_langevin_run(s.pos, s.vel, s.box, 1, **kw)  # warm (page in, list build)
    t = time.perf_counter()
    out = orc.md_langevin_run(s.pos, s.vel, s.box, nsteps, **kw)
    el = time.perf_counter() - t
    # the run includes one initial list build + force evaluation; count it as a step
    return (nsteps / el), orc.num_threads(), out


WORKLOADS = ("lj_slab", "lj_fluid", "charged_fluid", "charged_slab", "lj_slab_lfc")


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
        s = build_slab(mdf)
        rc, dt, T, gamma, shift, coul = 3.5, DT, TEMP, 1.0, 0.0, None
    elif w == "charged_fluid":
        s = mdf.systems.charged_fluid()
        rc, dt, T, gamma, shift = 3.0, 0.002, 1.0, 1.0, 0.0
        coul = dict(beta=0.95, K=(64, 64, 64), order=6)
    else:
        s = mdf.systems.charged_slab()
        rc, dt, T, gamma, shift = 3.0, 0.002, 1.0, 1.0, 0.0
        coul = dict(beta=None, K=(128, 128, 512), order=6)
    adaptive = w == "charged_slab"
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
        print(json.dumps(line), flush=True)
    return 0


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    import mdforce as mdf
    # the same seeded start, relaxation and cutoff lattice as the GPU arm; the
    # preparation is not timed (it runs on the device when one is present)
    s, lattice, rcinfo = equilibrate(mdf, build_slab(mdf), args.equil)
    from oracle import oracle as orc
    # bounded sample: estimate one step, cap the whole run at ~150 s
    sps0, cores, _ = cpu_baseline(s, lattice, 3)
    budget_steps = max(3, min(args.steps, int(150 * sps0)))
    sps, cores, out = cpu_baseline(s, lattice, budget_steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": sps, "unit": "steps/s", "n_gpus": args.gpus,
        "steps": budget_steps, "warmup": args.warmup, "ms_per_step": 1e3 / sps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "lj_slab_65536_npt", "n_atoms": s.n, "box": s.box.tolist(),
                   "rc": rcinfo, "skin": SKIN_SPEC, "dt": DT, "parallelism": "replicas"},
        "cpu_baseline": {"value": sps, "unit": "steps/s", "cores": cores, "kind": "port",
                         "sample": f"{budget_steps} Langevin NPT steps of the full 65536-atom slab "
                                   f"(oracle CPU FP64 cell+Verlet list LJ, OpenMP, skin {SKIN_SPEC})"},
        "e2e": {"value": sps, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
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

    s, lattice, rcinfo = equilibrate(mdf, build_slab(mdf), args.equil)
    stream = torch.cuda.Stream()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    # ---- mixed precision path (the headline value)
    use_graph = args.launch == "graph"
    sys_m, eng_m, sim_m = make_sim(mdf, s, 0, lattice, seed=1 + rank, use_graph=use_graph)
    sys_m.set_stream(stream.cuda_stream)
    sim_m.run(args.warmup)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    _, rebuilds0, _ = sim_m.counters()
    with Clocks(local) as clk:
        t_mixed = time_steps(torch, sim_m, stream, args.steps, flush, nvtx_range="timed")
    steps_done, rebuilds, flags = sim_m.counters()
    rebuilds_timed = rebuilds - rebuilds0
    value, t_max = replica_rate(torch, args.steps, t_mixed, world, "cuda")

    # back-to-back (warm L2) throughput of the same loop, for reference
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        a.record(stream)
        sim_m.run(args.steps)
        b.record(stream)
    torch.cuda.synchronize()
    warm_sps = args.steps / (a.elapsed_time(b) / 1e3)

    # ---- FP64 path, same steps
    fp64_sps = None
    if not args.no_fp64:
        sys_d, eng_d, sim_d = make_sim(mdf, s, 1, lattice, seed=1 + rank, use_graph=use_graph)
        sys_d.set_stream(stream.cuda_stream)
        sim_d.run(args.warmup)
        t64 = time_steps(torch, sim_d, stream, args.steps, flush)
        fp64_sps = args.steps / t64
        del sim_d, eng_d, sys_d

    # ---- dominant kernel: LJ forces, algorithmic bytes / CUDA-event duration
    t_lj, P, t_nl = time_lj_kernel(torch, mdf, sys_m, eng_m, sim_m, stream)
    N = s.n
    alg_bytes = N * 16 + N * 4 + P * 4 + N * 24  # positions, rcut, list indices, FP64 forces
    peak, peak_kind = measured_peak_hbm()
    achieved = alg_bytes / t_lj / 1e9
    rms_abs, rms_rel = force_error(mdf, s, lattice)

    # ---- end to end through the C ABI with host buffers
    e2e_steps = args.steps
    pin_pos = torch.from_numpy(np.ascontiguousarray(s.pos)).pin_memory()
    pin_vel = torch.from_numpy(np.ascontiguousarray(s.vel)).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sys_e, eng_e, sim_e = None, None, None
    sys_e = mdf.MDSystem(pin_pos.numpy(), s.box, vel=pin_vel.numpy(), precision=0)
    if lattice is None:
        sys_e.set_rcut(np.full(N, 2.5, np.float32))
    else:
        mdf.AssignRCut(lattice).assign(sys_e)
    eng_e = mdf.InteractionEngine(sys_e)
    eng_e.registNonBondedInteraction(1.0, 1.0, 0.0)
    lv = mdf.langevin_params(dt=DT, temperature=TEMP, gamma_t=1.0, tau_p=2.0, kappa_t=0.1,
                             p_ref=(0.0, 0.0, 0.0), npt_dirs=4, seed=1)
    sim_e = mdf.Simulation(sys_e, eng_e, skin=SKIN, cell_size=2.8, lv=lv, expansion=1.5)
    t_setup = time.perf_counter() - t0
    # one page-locked row per step: the device writes each step's energy /
    # virial / kinetic tensor there as the step ends; read once the run drains
    stat_rows = torch.zeros((e2e_steps, mdf.STAT_COUNT), dtype=torch.float64).pin_memory().numpy()
    sim_e.set_stats_ring(stat_rows)
    t1 = time.perf_counter()
    sim_e.run(e2e_steps)
    sys_e.synchronize()
    fin_pos = sys_e.positions()
    fin_f = sys_e.forces()
    t_e2e = time.perf_counter() - t1 + t_setup
    e2e_sps = e2e_steps / t_e2e
    h2d = (pin_pos.numel() + pin_vel.numel()) * 8 / e2e_steps
    d2h = mdf.STAT_COUNT * 8 + (fin_pos.size + fin_f.size) * 8 / e2e_steps
    if not np.isfinite(stat_rows).all() or not np.array_equal(stat_rows[-1], sys_e.stats()):
        raise RuntimeError("per-step statistics of the end-to-end run are missing or non-finite")

    # step1, LJ, step2 every step; bin, scan, scatter, order, gather, copy back,
    # list build per rebuild; the density deposit every 40 steps; 3 + 3*3 DFT
    # passes + 7 element-wise kernels per cutoff update (every 2000 steps)
    n_updates = (args.warmup + args.steps) // UPDATE_EVERY - args.warmup // UPDATE_EVERY
    # (direct launch: the 7 rebuild kernels are launched every step and return
    # early unless the device flag asks for a rebuild)
    rebuild_launches = 7 * (rebuilds_timed if use_graph else args.steps)
    launches = (3 * args.steps + rebuild_launches + args.steps // SAMPLE_EVERY + 22 * n_updates)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        n_cpu = 30
        sps_cpu, cores, _ = cpu_baseline(s, lattice, n_cpu)
        cpu = {"value": sps_cpu, "unit": "steps/s", "cores": cores, "kind": "port",
               "sample": f"{n_cpu} Langevin NPT steps of the full 65536-atom slab "
                         f"(oracle CPU FP64 cell+Verlet list LJ, OpenMP, skin {SKIN_SPEC})"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 pair math / f64 accumulation",
            "data": "synthetic",
            "config": {"workload": "lj_slab_65536_npt", "n_atoms": N, "box": s.box.tolist(),
                       "rc": rcinfo, "skin": SKIN, "dt": DT, "T": TEMP, "ensemble": "Langevin NPT Pzz=0",
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "flushed (256 MB write) between timed steps",
                       "start": f"random sequential addition, {args.equil} NVT relaxation steps"},
            "fp64_steps_per_s": fp64_sps,
            "speedup_vs_fp64": (value / world / fp64_sps) if fp64_sps else None,
            "warm_l2_steps_per_s": warm_sps,
            "force_rms_err_vs_fp64": {"abs": rms_abs, "rel": rms_rel},
            "list_rebuilds": rebuilds, "tau_per_day": value / world * DT * 86400,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profiled_traffic("k_lj_mixed"),
                         "kernel": "k_lj_mixed",
                         "kernel_us": t_lj * 1e6, "alg_bytes": alg_bytes, "peak_kind": peak_kind},
            "nlist_build_us": t_nl * 1e6,
            "e2e": {"value": e2e_sps, "unit": "steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps, "setup_s": t_setup,
                    "path": "MDSystem from pinned host arrays, Simulation.run(steps) with every step's "
                            "statistics written by the device into its own pinned host row, "
                            "positions and forces read back at the end"},
            "gpu_launches": launches,
            "list_rebuilds_timed": rebuilds_timed,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
