"""The archived slice files of the reference's rupture runs (test_problems/
truth/1 and truth/2: ``*.Hslice``, ``*.Vslice``, kept as
tests/golden/rupture_slices.npz) pin the slice layout and timing the slice
writer follows: per output time block 1's F(:, 1, :, 1:9) (horizontal, fixed
r) and F(:, :, 1, 1:9) (vertical, fixed s) as float32, q fastest, written
with the fault output before the step (the fields of t_(n-1)).  Both planes
are faces of the block that meet the fault edges, where the historical build
differs (see test_oracle_rupture.py); away from the fault face (q <= 14) the
oracle's planes match the files to a few float32 roundings after one step."""
import os

import numpy as np
import pytest

from cases import tpv5_case

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rupture_slices.npz")


def _case(oracle_lib, tag):
    if tag == "tpv5":
        return tpv5_case()
    from test_oracle_rupture_curv import archived_case
    return archived_case(oracle_lib)


@pytest.mark.parametrize("tag", ["tpv5", "tpv28"])
def test_slices_are_block1_planes_before_each_step(oracle_lib, tag):
    g = np.load(GOLDEN)
    H, V = g[tag + "_H"], g[tag + "_V"]          # (nsamp, 9, 21, 21)
    D = oracle_lib.OracleDomain(_case(oracle_lib, tag))
    for n in range(H.shape[0]):
        F = D.fields(0)                           # (9, ns, nr, nq)
        h, v = F[:, :, 0, :], F[:, 0, :, :]
        if n == 0:
            assert not H[0].any() and not V[0].any() and not h.any() and not v.any()
        else:
            for mine, arch in ((h, H[n]), (v, V[n])):
                err = np.abs(mine - arch)[:, :, :14].max() / np.abs(arch).max()
                assert err < 5e-6 if n == 1 else err < 1e-4, (n, err)
        D.run(1)
