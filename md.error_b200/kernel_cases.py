"""Runs one kernel family of libmdforce on a small case, for per-kernel ncu
captures.  The launches to capture sit inside the NVTX range "measure", so a
capture selects them with

    ncu --nvtx --nvtx-include "measure/" -k regex:<kernel> -c <n> ... \
        python md.error_b200/kernel_cases.py <case>

Cases:
  slab      the 65,536-atom slab start (tests/golden/slab65536_start.npz) under
            the Langevin NPT step in direct launches, 20 steps in the range:
            Langevin halves, LJ forces, the gated rebuild chain (cell sort, z
            order, list build)
  nlist     one cell-list rebuild (bin, scan, scatter, order, gather, copy
            back, z order) and one neighbour-list build on the slab start
            (radius rc_i + 0.6)
  lj        LJ forces over that list, 3 launches
  arc       AdaptRCut on the slab start: construction (the kernel tables),
            one deposit, update, assign and pressure correction
  errmap    the ik error map of the 20,736-atom charged fluid, K 32^3
  ikerr     the optiBasis functional: construction (the basis hats on the
            over-sampled grid) and one evaluation of 8 candidates, K 64^3
  bonded    harmonic bonds + angles on the LJ fcc crystal
  hspme     the Hermite-basis SPME of the charged fluid with all gradients, K 64^3
--precision 0 (mixed) or 1 (FP64) for slab, nlist, lj and bonded.
"""
import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402
import torch  # noqa: E402

import bench as B  # noqa: E402
import mdforce as mdf  # noqa: E402


def slab_system(prec):
    s = B.load_slab_start()
    sys_ = mdf.MDSystem(s.pos, s.box, vel=s.vel, precision=prec)
    mdf.AssignRCut(s.lattice).assign(sys_)
    return s, sys_


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["slab", "nlist", "lj", "arc", "errmap", "ikerr", "bonded", "hspme"])
    ap.add_argument("--precision", type=int, default=0)
    a = ap.parse_args()
    prec = a.precision
    nvtx = torch.cuda.nvtx
    if a.case == "slab":
        s, sys_ = slab_system(prec)
        eng = mdf.InteractionEngine(sys_)
        eng.registNonBondedInteraction(1.0, 1.0, 0.0)
        lv = mdf.langevin_params(dt=B.DT, temperature=B.TEMP, gamma_t=B.GAMMA_T, tau_p=B.TAU_P,
                                 kappa_t=B.KAPPA_T, p_ref=(0, 0, 0), npt_dirs=4, seed=1)
        sim = mdf.Simulation(sys_, eng, skin=B.SKIN, cell_size=2.8, lv=lv, expansion=1.5,
                             max_rcut=B.RC_MAX, use_graph=False)
        sim.run(20)
        torch.cuda.synchronize()
        nvtx.range_push("measure")
        sim.run(20)
        torch.cuda.synchronize()
        nvtx.range_pop()
    elif a.case in ("nlist", "lj"):
        s, sys_ = slab_system(prec)
        cl, nl = B.fitted_list(mdf, sys_)
        eng = mdf.InteractionEngine(sys_)
        eng.registNonBondedInteraction(1.0, 1.0, 0.0)
        eng.applyNonBondedInteraction(sys_, nl, with_stats=True)
        torch.cuda.synchronize()
        nvtx.range_push("measure")
        if a.case == "nlist":
            cl.rebuild()
            nl.rebuild(sys_, cl)
        else:
            for _ in range(3):
                eng.applyNonBondedInteraction(sys_, nl, with_stats=True)
        torch.cuda.synchronize()
        nvtx.range_pop()
    elif a.case == "arc":
        s, sys_ = slab_system(0)
        torch.cuda.synchronize()
        nvtx.range_push("measure")
        arc = mdf.AdaptRCutEstimator(sys_, refh=1.0, rcmin=B.RC_MIN, rcmax=B.RC_MAX, rcstep=B.RC_STEP)
        arc.deposite()
        arc.update(B.TARGET_PREC)
        arc.assign()
        arc.pressure_correction()
        torch.cuda.synchronize()
        nvtx.range_pop()
    elif a.case == "errmap":
        s = mdf.systems.charged_fluid()
        sys_ = mdf.MDSystem(s.pos, s.box, charge=s.charge, precision=1)
        em = mdf.ErrorEstimate_SPME_Ik((32, 32, 32), s.box, 0.95, 6)
        nvtx.range_push("measure")
        em.deposit(sys_)
        em.rms(1.0)
        torch.cuda.synchronize()
        nvtx.range_pop()
    elif a.case == "ikerr":
        c = np.tile(mdf.optibasis.bspline_initial_basis(2.0, 16, 4), (8, 1))
        torch.cuda.synchronize()
        nvtx.range_push("measure")
        f = mdf.optibasis.IkErrorGPU(2.0, 16, 0.95, (64, 64, 64), 20736.0, 20736, [30.0, 30.0, 30.0], l_cut=10)
        f.evaluate(c)
        torch.cuda.synchronize()
        nvtx.range_pop()
    elif a.case == "bonded":
        s = mdf.systems.lj_fluid_fcc()
        sys_ = mdf.MDSystem(s.pos, s.box, precision=prec)
        eng = mdf.InteractionEngine(sys_)
        n = s.n - s.n % 4
        eng.setBonds(np.array([[i, i + 1] for i in range(0, n, 2)], np.int32), mdf.BOND_HARMONIC, (100.0, 1.0))
        eng.setAngles(np.array([[i, i + 1, i + 2] for i in range(0, n - 2, 4)], np.int32),
                      mdf.ANGLE_HARMONIC, (50.0, 1.5))
        eng.clearInteraction()
        eng.applyBondedInteraction(sys_)
        torch.cuda.synchronize()
        nvtx.range_push("measure")
        for _ in range(3):
            eng.clearInteraction()
            eng.applyBondedInteraction(sys_)
        torch.cuda.synchronize()
        nvtx.range_pop()
    elif a.case == "hspme":
        s = mdf.systems.charged_fluid()
        q = torch.tensor(s.charge, dtype=torch.float64, device="cuda")
        r = torch.tensor(s.pos, dtype=torch.float64, device="cuda")
        hs = mdf.optibasis.HermiteSPME(s.n, (64, 64, 64), s.box, 0.95, 3.0, 16)
        c = torch.tensor(np.tile(mdf.optibasis.bspline_initial_basis(3.0, 16, 6), (2, 1)), device="cuda")
        nvtx.range_push("measure")
        hs.energy(q, r, c, forces=True, grads=True)
        torch.cuda.synchronize()
        nvtx.range_pop()
    torch.cuda.synchronize()
    print("ok", a.case)


if __name__ == "__main__":
    main()
