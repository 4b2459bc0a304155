"""Builds tests/golden/arc_t085_n16000.json from the reference's published
adaptive-cutoff profiles of the 16000-atom slab at T* = 0.85, target 0.0045
(shortRange.inhomo/alltext/writeDown/fig/t0.85-n16000-adapt-e0.0045/
a.density.x.out, a.rcut.x.out, a.error.x.out).  Run in a tree where the
reference is present (MDERROR_REFERENCE); the JSON it writes is committed."""
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from oracle.refpath import reference_root  # noqa: E402

REF = sys.argv[1] if len(sys.argv) > 1 else reference_root()
if not REF:
    sys.exit("reference tree not found: set MDERROR_REFERENCE or pass its path")
D = os.path.join(REF, "shortRange.inhomo/alltext/writeDown/fig/t0.85-n16000-adapt-e0.0045")


def cols(name):
    xs, ys = [], []
    for line in open(os.path.join(D, name)):
        p = line.split()
        if len(p) >= 2 and not line.startswith("#"):
            xs.append(float(p[0]))
            ys.append(float(p[1]))
    return xs, ys


dx, dy = cols("a.density.x.out")
rx, ry = cols("a.rcut.x.out")
ex, ey = cols("a.error.x.out")
out = {
    "source": "shortRange.inhomo/alltext/writeDown/fig/t0.85-n16000-adapt-e0.0045/a.{density,rcut,error}.x.out",
    "box": [150.0, 21.0, 21.0],  # conf.16000.gro / main.tex:705-740
    "target": 0.0045,
    "density_x": dx, "density": dy,
    "rcut_x": rx, "rcut": ry,
    "error_x": ex, "error": ey,
}
json.dump(out, open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "arc_t085_n16000.json"), "w"))
print("wrote", len(dx), len(rx), len(ex))
