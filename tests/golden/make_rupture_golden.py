"""Write tests/golden/tpv5_cartesian_truth.npz, tpv28_curvilinear_truth.npz
and rupture_slices.npz from the reference's archived rupture output:
test_problems/truth/1 (the TPV5 two-block Cartesian problem of
test_problems/test_rup_cart_fric.in) and test_problems/truth/2 (the TPV28
two-block curvilinear problem of test_problems/test_rup_curv_fric.in), fault
files, stations and the block-1 slices (.Hslice / .Vslice: 46 samples x 9 x
21 x 21 float32, q fastest).

The archived files are float32 in the layout python/read_binary.py reads:
46 samples x ncomp x 21 x 21 (y fastest).  Only the first NSAMP samples are
kept: later samples carry the discrepancy at the fault edges described in
test_oracle_rupture.py.  The seismogram files (text, 6 decimals) are kept for
the first NSEIS samples.

Run in a tree where the reference is mounted:
    python tests/golden/make_rupture_golden.py /path/to/reference
"""
import os
import sys

import numpy as np

NSAMP = 4
NSEIS = 12
FILES = (("S", 4), ("Svel", 3), ("Uface", 9), ("Vface", 9), ("Uhat", 6), ("Vhat", 6), ("trup", 1))


def one(ref: str, truth: str, stem: str, fname: str) -> str:
    base = os.path.join(ref, "test_problems", "truth", truth, stem)
    out = {}
    for name, nc in FILES:
        a = np.fromfile(base + "_interface." + name, dtype=np.float32).reshape(46, nc, 21, 21)
        out[name] = a[:NSAMP].copy()
    out["seis_block1"] = np.loadtxt(base + "_21_11_11.dat")[:NSEIS]
    out["seis_block2"] = np.loadtxt(base + "_1_11_11.dat")[:NSEIS]
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), fname)
    np.savez_compressed(path, **out)
    return path


def slices(ref: str) -> str:
    out = {}
    for tag, truth, stem in (("tpv5", "1", "test_rup_cart_fric"), ("tpv28", "2", "test_rup_curv_fric")):
        base = os.path.join(ref, "test_problems", "truth", truth, stem)
        for kind in ("H", "V"):
            a = np.fromfile(base + "." + kind + "slice", dtype=np.float32).reshape(46, 9, 21, 21)
            out[tag + "_" + kind] = a[:NSAMP].copy()
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rupture_slices.npz")
    np.savez_compressed(path, **out)
    return path


def main(ref: str) -> str:
    return "\n".join([one(ref, "1", "test_rup_cart_fric", "tpv5_cartesian_truth.npz"),
                      one(ref, "2", "test_rup_curv_fric", "tpv28_curvilinear_truth.npz"),
                      slices(ref)])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_rupture_golden.py <reference project root>")
    print(main(sys.argv[1]))
