#!/usr/bin/env python3
"""Builds tests/golden/slab65536_start.npz, the start state of the 65,536-atom
liquid-vapour slab workload (40 x 40 x 160 sigma, liquid rho* 0.78 for
|z - 80| < 24.84, vapour 0.02), shared by bench.py's two arms and by the
headline-scale parity tests:

1. the seeded random-sequential-addition start (md_synth_slab, host code,
   0.8 sigma minimum separation, seed 0) with Maxwell velocities at T* 0.85;
2. 4000 steps of Langevin NVT relaxation (gamma 2, T* 0.85, dt 0.005,
   uniform rc 2.5, skin 0.3) by the CPU FP64 oracle, in chunks of 40 steps;
3. the density profile on 1-sigma bins (41 x 41 x 161), sampled every 40
   steps over the second half of the relaxation;
4. the adaptive cutoff lattice from that profile by the reference's own
   AdaptRCut (ENG/src/AdaptRCut.cu, built in oracle/_ref) at targetPrec 0.02
   (ENG/app/lj.nhc-xtc.cu:57), rc 2.5..5.0 step 0.5, checked equal to the
   oracle's restatement.

Nothing here runs on a GPU.  Positions and velocities are stored in binary32
(both arms start from exactly these values).  Run once, where the reference
tree was present when oracle/_ref was built:

    python tests/golden/make_slab_start.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "md.error_b200"))

from oracle import oracle as orc  # noqa: E402
from mdforce import systems  # noqa: E402  (host-only generators, no device use)

OUT = os.path.join(HERE, "slab65536_start.npz")
RELAX, CHUNK, SEED0 = 4000, 40, 12345
TARGET, RCMIN, RCMAX, RCSTEP = 0.02, 2.5, 5.0, 0.5


def main():
    if not orc.ref_available("libref_arc.so"):
        sys.exit("oracle/_ref/libref_arc.so is missing: build oracle/ref with the reference tree present")
    s = systems.lj_slab()
    n_bins = orc.dp_bins(s.box, 1.0)
    pos, vel = s.pos.copy(), s.vel.copy()
    rc = np.full(s.n, 2.5, np.float32)
    prof = np.zeros(n_bins, np.float64)
    samples = 0
    t0 = time.time()
    for c in range(RELAX // CHUNK):
        out = orc.md_langevin_run(pos, vel, s.box, CHUNK, dt=0.005, temperature=0.85, gamma_t=2.0, skin=0.3,
                                  rcut=rc, seed=SEED0 + c)
        if out["status"] != 0:
            sys.exit(f"oracle relaxation failed at chunk {c}: status {out['status']}")
        pos, vel = out["pos"], out["vel"]
        if (c + 1) * CHUNK > RELAX // 2:
            orc.dp_deposit(pos.astype(np.float32), s.box, n_bins, prof)
            samples += 1
        if c % 10 == 0:
            print(f"chunk {c}: {time.time() - t0:.0f} s, rebuilds {out['rebuilds']}", flush=True)
    dv = float(np.prod(s.box / np.array(n_bins)))
    rho = prof / (samples * dv)
    ref = orc.ref_adapt_rcut(s.box, n_bins, RCMIN, RCMAX, RCSTEP, rho, TARGET)
    mine = orc.adapt_rcut(s.box, n_bins, np.arange(RCMIN, RCMAX + 1e-9, RCSTEP), rho, TARGET)
    if not np.array_equal(ref["rcut"], mine["rcut"]):
        sys.exit("oracle and reference AdaptRCut disagree on the lattice")
    lattice = ref["rcut"].astype(np.float32)
    # positions wrapped into the box
    pos = pos - np.floor(pos / s.box) * s.box
    np.savez_compressed(OUT, pos=pos.astype(np.float32), vel=vel.astype(np.float32), box=s.box,
                        lattice=lattice, samples=np.int32(samples), relax_steps=np.int32(RELAX))
    counts = {float(v): int((lattice == v).sum()) for v in np.unique(lattice)}
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes); lattice {n_bins}, bins per rc {counts}")


if __name__ == "__main__":
    main()
