"""Curvilinear block meshes by transfinite interpolation, built on the device.

The reference generates a curvilinear block from its six boundary surfaces
(src/grid.f90:473-1909, Curve_Grid_3D3): the two q-faces carry the fault or
interface profile, the r- and s-faces follow from 2-D transfinite
interpolation of their edge curves (Gen_Surf_Mesh, :2420-2457), and the
volume from 3-D transfinite interpolation (Gen3_Curve_Mesh, :2292-2418).
Here the six surfaces (2-D, cheap) are built on the host and the volume --
the O(n^3) part -- by the library's ``wql3d_tfi_grid`` kernel.

Surface layout handed to the kernel, x / y / z components each:
left / right (q = 0 / 1): (ns, nr); top / bottom (r = 0 / 1): (ns, nq);
front / back (s = 0 / 1): (nr, nq) -- numpy C order, the first index slowest.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Dict, Tuple

import numpy as np


def gen_surf_mesh(XL, XR, XB, XT, YL, YR, YB, YT):
    """2-D transfinite interpolation of a face from its four edge curves
    (src/grid.f90:2420-2457).  XL/XR/YL/YR have my entries, XB/XT/YB/YT mx;
    returns X, Y of shape (my, mx) (second reference index slowest)."""
    mx, my = len(XB), len(XL)
    q = (np.arange(mx) * (1.0 / (mx - 1)))[None, :]
    r = (np.arange(my) * (1.0 / (my - 1)))[:, None]

    def one(L, R, B, T):
        L, R, B, T = (np.asarray(a, dtype=np.float64) for a in (L, R, B, T))
        return ((1.0 - q) * L[:, None] + q * R[:, None] + (1.0 - r) * B[None, :] + r * T[None, :]
                - (1.0 - q) * (1.0 - r) * L[0] - q * (1.0 - r) * R[0] - r * (1.0 - q) * T[0] - (r * q) * T[-1])

    return one(XL, XR, XB, XT), one(YL, YR, YB, YT)


def block_surfaces(nqrs: Tuple[int, int, int], aqrs, bqrs, lc: float, rc: float,
                   profile: str = "analytical_test_problem") -> Dict[str, np.ndarray]:
    """The six boundary surfaces of a block (src/grid.f90:587-1150) for the
    profile of its q-faces: 'flat', or 'analytical_test_problem' (the
    curvilinear rupture test: Gaussian bump plus sine pattern of 0.1 km
    on the q-face that carries lc / rc).  Returns {face: (3, d1, d0)}."""
    mx, my, mz = nqrs
    ax, ay, az = aqrs
    bx, by, bz = bqrs
    hy = (by - ay) / (my - 1)
    hz = (bz - az) / (mz - 1)
    ys = ay + np.arange(my) * hy
    zs = az + np.arange(mz) * hz
    # q-faces: (Y, Z) by 2-D interpolation of straight edges, X from the
    # profile; arrays below are indexed [j, k] (r, s) like the reference's
    Yq, Zq = gen_surf_mesh(np.full(mz, ay), np.full(mz, by), ys, ys, zs, zs, np.full(my, az), np.full(my, bz))
    YL, ZL = Yq.T.copy(), Zq.T.copy()
    YR, ZR = Yq.T.copy(), Zq.T.copy()
    if profile == "analytical_test_problem":
        def bump(Y, Z, c):
            return (0.1 * c * np.exp(-((1.0 * Y - 0.5 * (ay + by)) ** 2 + 1.0 * (Z - 0.5 * (az + bz)) ** 2) / 0.025)
                    + 0.1 * c * np.sin(2.0 / (by - ay) * math.pi * Y) * np.sin(2.0 / (bz - az) * math.pi * Z))
        XL = ax + bump(YL, ZL, rc)
        XR = bx + bump(YR, ZR, lc)
    elif profile == "flat":
        XL = np.full_like(YL, ax)
        XR = np.full_like(YR, bx)
    else:
        raise ValueError("unknown profile %r" % profile)
    ii = np.arange(mx)

    def line(a, b):
        return a + ii * ((b - a) / (mx - 1))

    # front (k = 1) and back (k = mz) faces, z constant; results [j, i]
    Xf, Yf = gen_surf_mesh(XL[:, 0], XR[:, 0], line(XL[0, 0], XR[0, 0]), line(XL[-1, 0], XR[-1, 0]),
                           YL[:, 0], YR[:, 0], line(YL[0, 0], YR[0, 0]), line(YL[-1, 0], YR[-1, 0]))
    Xb, Yb = gen_surf_mesh(XL[:, -1], XR[:, -1], line(XL[0, -1], XR[0, -1]), line(XL[-1, -1], XR[-1, -1]),
                           YL[:, -1], YR[:, -1], line(YL[0, -1], YR[0, -1]), line(YL[-1, -1], YR[-1, -1]))
    Zf = np.full_like(Xf, az)
    Zb = np.full_like(Xb, bz)
    # top (j = 1) and bottom (j = my) faces, y constant; results [k, i]
    Xt, Zt = gen_surf_mesh(XL[0, :], XR[0, :], line(XL[0, 0], XR[0, 0]), line(XL[0, -1], XR[0, -1]),
                           ZL[0, :], ZR[0, :], Zf[0, :], Zb[0, :])
    Xo, Zo = gen_surf_mesh(XL[-1, :], XR[-1, :], line(XL[-1, 0], XR[-1, 0]), line(XL[-1, -1], XR[-1, -1]),
                           ZL[-1, :], ZR[-1, :], Zf[-1, :], Zb[-1, :])
    Yt = np.full_like(Xt, ay)
    Yo = np.full_like(Xo, by)
    return {
        "left": np.stack([XL.T, YL.T, ZL.T]), "right": np.stack([XR.T, YR.T, ZR.T]),   # (3, mz, my)
        "top": np.stack([Xt, Yt, Zt]), "bottom": np.stack([Xo, Yo, Zo]),              # (3, mz, mx)
        "front": np.stack([Xf, Yf, Zf]), "back": np.stack([Xb, Yb, Zb]),              # (3, my, mx)
    }


FACES = ("left", "right", "top", "bottom", "front", "back")


def pack_surfaces(surf: Dict[str, np.ndarray]) -> np.ndarray:
    """The six surfaces concatenated in FACES order, each (3, d1, d0)."""
    return np.ascontiguousarray(np.concatenate([np.ascontiguousarray(surf[f]).ravel() for f in FACES]))


def tfi_grid(surf: Dict[str, np.ndarray], nqrs: Tuple[int, int, int]) -> np.ndarray:
    """Coordinates (3, ns, nr, nq) of the block by 3-D transfinite
    interpolation on the device (Gen3_Curve_Mesh, src/grid.f90:2292-2418)."""
    from . import _lib
    nq, nr, ns = nqrs
    faces = pack_surfaces(surf)
    out = np.zeros((3, ns, nr, nq))
    _lib.check(_lib.load().wql3d_tfi_grid(faces.ctypes.data_as(_lib.dp), nq, nr, ns,
                                          out.ctypes.data_as(_lib.dp)), "wql3d_tfi_grid")
    return out
