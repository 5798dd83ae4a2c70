"""The try_traditional_cartesian_rhs seam (wql3d_traditional_cartesian_rhs) on
the caller's device arrays: the strict-interior rates of
cartesian_elastic_o6_interior_kernel (src/traditional_cartesian_rhs_openacc.f90)
for arrays with ghost layers, equal bit for bit to a numpy evaluation of the
same expressions in the same order (no fused multiply-add on either side), and
the points outside the box untouched."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _numpy_rates(F, R, MX, MY, MZ, MAT, box, h):
    """The reference kernel's loop body over the box, vectorised: F, R are
    (9, n3, n2, n1), the metrics (nm, n3, n2, n1), MAT (nmat, n3, n2, n1);
    box = (xlo, xhi, ylo, yhi, zlo, zhi) 1-based."""
    xlo, xhi, ylo, yhi, zlo, zhi = box
    X = slice(xlo - 1, xhi)
    Y = slice(ylo - 1, yhi)
    Z = slice(zlo - 1, zhi)
    R = R.copy()
    mx, my, mz = MX[0][Z, Y, X], MY[1][Z, Y, X], MZ[2][Z, Y, X]
    dfx = [np.zeros_like(mx) for _ in range(9)]
    dfy = [np.zeros_like(mx) for _ in range(9)]
    dfz = [np.zeros_like(mx) for _ in range(9)]
    for s, coef in ((1, 0.75), (2, -0.15), (3, 1.0 / 60.0)):
        cx, cy, cz = coef / h[0], coef / h[1], coef / h[2]
        for c in range(9):
            f = F[c]
            dfx[c] = dfx[c] + (mx * cx) * (f[Z, Y, slice(xlo - 1 + s, xhi + s)] - f[Z, Y, slice(xlo - 1 - s, xhi - s)])
            dfy[c] = dfy[c] + (my * cy) * (f[Z, slice(ylo - 1 + s, yhi + s), X] - f[Z, slice(ylo - 1 - s, yhi - s), X])
            dfz[c] = dfz[c] + (mz * cz) * (f[slice(zlo - 1 + s, zhi + s), Y, X] - f[slice(zlo - 1 - s, zhi - s), Y, X])
    lam, mu, rho = MAT[0][Z, Y, X], MAT[1][Z, Y, X], MAT[2][Z, Y, X]
    a1 = 1.0 / rho
    a2 = lam + 2.0 * mu
    r = [R[c][Z, Y, X] for c in range(9)]
    r[0] = r[0] + a1 * ((dfx[3] + dfy[6]) + dfz[7])
    r[1] = r[1] + a1 * ((dfx[6] + dfy[4]) + dfz[8])
    r[2] = r[2] + a1 * ((dfx[7] + dfy[8]) + dfz[5])
    r[3] = (r[3] + a2 * dfx[0]) + lam * (dfy[1] + dfz[2])
    r[4] = (r[4] + a2 * dfy[1]) + lam * (dfx[0] + dfz[2])
    r[5] = (r[5] + a2 * dfz[2]) + lam * (dfx[0] + dfy[1])
    r[6] = r[6] + mu * (dfy[0] + dfx[1])
    r[7] = r[7] + mu * (dfz[0] + dfx[2])
    r[8] = r[8] + mu * (dfz[1] + dfy[2])
    for c in range(9):
        R[c][Z, Y, X] = r[c]
    return R


def test_seam_rates_equal_reference_expressions(wql3d_lib):
    import torch
    from waveqlab3d_q_gpu_b200 import _lib
    rng = np.random.default_rng(5)
    n = (24, 21, 19)                        # n1, n2, n3 with 3 ghost layers around 18 x 15 x 13 points
    shape = (n[2], n[1], n[0])
    F = rng.standard_normal((9,) + shape)
    R0 = rng.standard_normal((9,) + shape)
    MX = 1.0 + 0.1 * rng.random((3,) + shape)
    MY = 1.0 + 0.1 * rng.random((3,) + shape)
    MZ = 1.0 + 0.1 * rng.random((3,) + shape)
    MAT = np.stack([30 + rng.random(shape), 20 + rng.random(shape), 2.5 + 0.1 * rng.random(shape)])
    h = (1.0 / 17, 1.0 / 14, 1.0 / 12)
    box = (4 + 6, n[0] - 3 - 6, 4 + 6, n[1] - 3 - 6, 4 + 6, n[2] - 3 - 6)
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (F, R0, MX, MY, MZ, MAT)]
    L = _lib.load()
    rc = L.wql3d_traditional_cartesian_rhs(*[t.data_ptr() for t in dev], n[0], n[1], n[2], 3, 3, *box, *h, None)
    assert rc == 0
    torch.cuda.synchronize()
    got = dev[1].cpu().numpy()
    ref = _numpy_rates(F, R0, MX, MY, MZ, MAT, box, h)
    assert np.array_equal(got, ref)
    xlo, xhi, ylo, yhi, zlo, zhi = box
    inside = np.zeros(shape, bool)
    inside[zlo - 1:zhi, ylo - 1:yhi, xlo - 1:xhi] = True
    assert np.array_equal(got[:, ~inside], R0[:, ~inside])
    assert not np.array_equal(got[:, inside], R0[:, inside])
    # a box that leaves fewer than three stencil points inside the arrays is refused
    bad = (3, n[0] - 3, 4, n[1] - 3, 4, n[2] - 3)
    assert L.wql3d_traditional_cartesian_rhs(*[t.data_ptr() for t in dev], n[0], n[1], n[2], 3, 3, *bad, *h,
                                             None) == -1   # WQL3D_EINVAL
