#!/usr/bin/env python3
"""Generate tests/golden/ikerror_cases.json: values and basis gradients of the
optiBasis ik-SPME force-error functional computed by the reference's own
Python (optiBasis/IkError.py HermiteLossFunc / HermiteLossFunc_Bound0, with
optiBasis/HatComput.py and optiBasis/Hermite.py), imported from the reference
tree.  Run once where the reference tree is present:

    python tests/golden/make_ikerror_golden.py [/path/to/reference]

The reference writes basis.step.out into its working directory, so the
script runs it from a temporary directory."""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def water_like(L):
    """q2 and atom count of the reference's water-like system
    (optiBasis/compute_basis.py:70-72)."""
    vol = float(np.prod(L))
    return 33.456 * vol * (0.8476 ** 2 + 2 * 0.4238 ** 2), 33.456 * vol * 3


def main():
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    from oracle.refpath import reference_root
    ref = sys.argv[1] if len(sys.argv) > 1 else reference_root()
    if not ref:
        sys.exit("reference tree not found: set MDERROR_REFERENCE or pass its path")
    sys.path.insert(0, os.path.join(ref, "optiBasis"))
    from Region import Region
    from Bspline import Bspline
    from IkError import HermiteLossFunc, HermiteLossFunc_Bound0
    import basis_common as bc

    cases = [
        # the reference's own __main__ defaults (optiBasis/IkError.py:262-307)
        dict(name="main_k32", KK=[32, 32, 32], L=[3.72412] * 3, beta=3.5, CC=2, nbin=10, l_cut=10,
             bound0=False, q2=(0.8476 ** 2 + 0.4238 ** 2 * 2) * 1728, natoms=3 * 1728, order=4),
        dict(name="aniso", KK=[16, 12, 20], L=[3.0, 2.5, 4.0], beta=3.0, CC=2, nbin=4, l_cut=4,
             bound0=False, order=4),
        dict(name="bound0", KK=[16, 16, 16], L=[1.8621] * 3, beta=3.5, CC=2, nbin=6,
             l_cut=bc.estimate_l_cut(2, 6, True), bound0=True, order=4),
    ]
    out = []
    cwd = os.getcwd()
    tmp = tempfile.mkdtemp()
    os.chdir(tmp)
    try:
        for c in cases:
            L = np.array(c["L"], dtype=float)
            if "q2" not in c:
                c["q2"], c["natoms"] = water_like(L)
            region = Region(L)
            cls = HermiteLossFunc_Bound0 if c["bound0"] else HermiteLossFunc
            loss = cls(c["CC"], c["nbin"], c["beta"], c["KK"], c["q2"], c["natoms"], region, l_cut=c["l_cut"])
            # B-spline initial basis (optiBasis/compute_basis.py:80-93)
            bstep = c["CC"] / float(c["nbin"])
            bs = Bspline(c["order"])
            bx = np.arange(0, c["CC"] + .5 * bstep, bstep)
            bv_, bd_ = bs(bx), bs.deriv(bx)
            bv, bd = bv_[1:] / bv_[0], bd_[1:] / bv_[0]
            if c["bound0"]:
                bv, bd = np.delete(bv, -1), np.delete(bd, -1)
            vv0 = bc.pack_v_d(bv, bd)
            rng = np.random.default_rng(7)
            vv1 = vv0 + rng.normal(0.0, 0.1, vv0.shape)
            evals = []
            for vv in (vv0, vv1):
                val = float(loss.value(vv))
                der = np.asarray(loss.deriv(vv), dtype=float)
                evals.append(dict(vv=vv.tolist(), value=val, deriv=der.tolist()))
            # the hat of the current basis along axis 0 at |k| <= K/2 + l_cut K
            kmax = c["KK"][0] // 2 + c["l_cut"] * c["KK"][0]
            hat0 = np.asarray(loss.hhc[0].get_value_buff()[: kmax + 1], dtype=float)
            rec = dict(c, evals=evals, hat_axis0_last=hat0.tolist(),
                       over_smpl=int(400 * (c["nbin"] / c["CC"])))
            out.append(rec)
            print(f"\n{c['name']}: value {evals[0]['value']:.12e} / {evals[1]['value']:.12e}", file=sys.stderr)
    finally:
        os.chdir(cwd)
    with open(os.path.join(HERE, "ikerror_cases.json"), "w") as f:
        json.dump(dict(source="optiBasis/IkError.py HermiteLossFunc(_Bound0).value/deriv", cases=out), f)


if __name__ == "__main__":
    main()
