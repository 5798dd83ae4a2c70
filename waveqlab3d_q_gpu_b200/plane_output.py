"""Plane and slice writers in the reference's binary layouts.

:class:`PlaneOutput` follows src/plane_output.f90: one file per plane,
``<domain>_<name>_block<b>.plane`` (``<domain>_plane_block<b>.plane`` when the
name is empty), opened with a header of int32 version 1, int32 axis id (1:
``yz``/``rs``, 2: ``xz``/``qs``, 3: ``xy``/``qr``), int32 n1, int32 n2,
float64 coordinate, int32 fixed index; then for every written call float64
t and the velocities vx, vy, vz as float64 n1 x n2 arrays, the first index
fastest (write_one_plane, :271-340).  A plane ``yz`` / ``xz`` / ``xy`` sits at
the index whose grid coordinate x / y / z is nearest to the requested one over
the whole block, the first such point in storage order (find_best_fixed_index,
:495-530), and is dropped when the coordinate lies outside the block; ``rs`` /
``qs`` / ``qr`` take the coordinate as a 1-based logical index.  Each plane
writes on every stride-th call (its own step counter).

:class:`SliceOutput` follows src/slice_output.f90: ``<name>.Hslice`` holds
F(:, locationH, :, 1:9) and ``<name>.Vslice`` F(:, :, locationV, 1:9) of
block 1 as float32, q fastest, per written call (write_slice, :79-94).

The planes come off the device through :meth:`Domain.plane` (a gather kernel
and one copy of the plane), not through a field readback.
"""
from __future__ import annotations

import os
import struct
from typing import List, Optional, Sequence

import numpy as np

# axis -> (axis id, fixed direction 1..3, logical coordinate)
AXES = {"yz": (1, 1, False), "xz": (2, 2, False), "xy": (3, 3, False),
        "rs": (1, 1, True), "qs": (2, 2, True), "qr": (3, 3, True)}


def block_coords(block) -> np.ndarray:
    """(3, ns, nr, nq) physical coordinates of a block: its mesh, or the
    Cartesian grid of aqrs .. bqrs."""
    if block.coords is not None:
        return np.asarray(block.coords, dtype=np.float64)
    nq, nr, ns = block.nqrs
    ax = [np.linspace(block.aqrs[k], block.bqrs[k], n) for k, n in enumerate((nq, nr, ns))]
    x = np.broadcast_to(ax[0][None, None, :], (ns, nr, nq))
    y = np.broadcast_to(ax[1][None, :, None], (ns, nr, nq))
    z = np.broadcast_to(ax[2][:, None, None], (ns, nr, nq))
    return np.stack([x, y, z])


def fixed_index(block, axis: str, coord: float) -> Optional[int]:
    """1-based index of the plane (init_one_plane, src/plane_output.f90:87-181),
    None when the plane is not in the block."""
    axis_id, fdir, logical = AXES[axis]
    n = block.nqrs[fdir - 1]
    if logical:
        i = int(round(coord))
        if abs(coord - i) > 1.0e-6 or i < 1 or i > n:
            return None
        return i
    X = block_coords(block)[fdir - 1]
    if coord < X.min() or coord > X.max():
        return None
    k = int(np.argmin(np.abs(X - coord)))   # first minimum in storage order (q fastest)
    ks, rem = divmod(k, X.shape[1] * X.shape[2])
    kr, kq = divmod(rem, X.shape[2])
    return (kq, kr, ks)[fdir - 1] + 1


class Plane:
    """One plane of one block."""

    def __init__(self, domain, block: int, axis: str, coord: float, name: str = "", stride: int = 1,
                 directory: str = ".", domain_name: str = "data"):
        if axis not in AXES:
            raise ValueError("plane axis must be one of %s" % ", ".join(AXES))
        self.domain, self.block = domain, block
        self.axis_id, self.fdir, _ = AXES[axis]
        self.coord = float(coord)
        self.stride = max(1, int(stride))
        self.counter = 0
        blk = domain.blocks[block]
        self.index = fixed_index(blk, axis, coord)
        self.file = None
        if self.index is None:
            return
        nq, nr, ns = blk.nqrs
        self.n1 = nr if self.fdir == 1 else nq
        self.n2 = nr if self.fdir == 3 else ns
        fname = (f"{domain_name}_{name}_block{block + 1}.plane" if name.strip()
                 else f"{domain_name}_plane_block{block + 1}.plane")
        if directory.strip() and directory.strip() != ".":
            os.makedirs(directory, exist_ok=True)
            fname = os.path.join(directory, fname)
        self.path = fname
        self.file = open(fname, "wb")
        self.file.write(struct.pack("<iiiidi", 1, self.axis_id, self.n1, self.n2, self.coord, self.index))

    @property
    def active(self) -> bool:
        return self.file is not None

    def write(self, t: float):
        if self.file is None:
            return
        self.counter += 1
        if (self.counter - 1) % self.stride != 0:
            return
        v = self.domain.plane(self.block, self.fdir, self.index, 0, 3)   # (3, n2, n1)
        self.file.write(struct.pack("<d", float(t)))
        np.ascontiguousarray(v, dtype=np.float64).tofile(self.file)

    def close(self):
        if self.file is not None:
            self.file.close()
            self.file = None


class PlaneOutput:
    """&plane_output_list of one domain: the listed planes of every block
    (write_plane_output is called per block, src/domain.f90:775-776)."""

    def __init__(self, domain, axes: Sequence[str], coords: Sequence[float], names: Optional[Sequence[str]] = None,
                 stride: int = 1, directory: str = ".", domain_name: str = "data"):
        names = list(names) if names is not None else [""] * len(axes)
        self.planes: List[Plane] = []
        for b in range(domain.nblocks):
            for ax, c, nm in zip(axes, coords, names):
                self.planes.append(Plane(domain, b, ax, c, nm, stride, directory, domain_name))
        self.domain = domain

    def write(self):
        for p in self.planes:
            p.write(self.domain.t)

    def close(self):
        for p in self.planes:
            p.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class SliceOutput:
    """&slice_list: horizontal (fixed r = locationH) and vertical (fixed s =
    locationV) slices of block 1, all nine fields, float32."""

    def __init__(self, domain, name: str, horz: bool = False, vert: bool = False, locationH: int = 1,
                 locationV: int = 1):
        self.domain = domain
        self.locationH, self.locationV = int(locationH), int(locationV)
        self.H = open(name + ".Hslice", "wb") if horz else None
        self.V = open(name + ".Vslice", "wb") if vert else None

    def write(self):
        if self.H is not None:
            np.ascontiguousarray(self.domain.plane(0, 2, self.locationH), dtype=np.float32).tofile(self.H)
        if self.V is not None:
            np.ascontiguousarray(self.domain.plane(0, 3, self.locationV), dtype=np.float32).tofile(self.V)

    def close(self):
        for f in (self.H, self.V):
            if f is not None:
                f.close()
        self.H = self.V = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def read_plane(path: str):
    """(header dict, times, v) of a .plane file; v is (nt, 3, n2, n1)."""
    with open(path, "rb") as f:
        raw = f.read()
    version, axis_id, n1, n2, coord, fixed = struct.unpack_from("<iiiidi", raw, 0)
    off = struct.calcsize("<iiiidi")
    rec = 8 + 3 * n1 * n2 * 8
    nt = (len(raw) - off) // rec
    t = np.zeros(nt)
    v = np.zeros((nt, 3, n2, n1))
    for k in range(nt):
        o = off + k * rec
        t[k] = struct.unpack_from("<d", raw, o)[0]
        v[k] = np.frombuffer(raw, dtype=np.float64, count=3 * n1 * n2, offset=o + 8).reshape(3, n2, n1)
    return {"version": version, "axis": axis_id, "n1": n1, "n2": n2, "coord": coord, "index": fixed}, t, v


def read_slice(path: str, nq: int, n2: int) -> np.ndarray:
    """A .Hslice (n2 = ns) or .Vslice (n2 = nr) file as (nt, 9, n2, nq)."""
    a = np.fromfile(path, dtype=np.float32)
    return a.reshape(-1, 9, n2, nq)
