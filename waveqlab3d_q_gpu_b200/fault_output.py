"""Fault output files in the reference's binary layout.

The reference writes, at stage 1 of every step n with mod(n - 1, w_stride)
== 0 (src/time_step.f90:137), eight files ``<name>_interface.<field>``
(src/fault_output.f90:13-122, called from write_fault_output /
write_hat_output, src/domain.f90:782-845): per output time one float32
record of ncomp x ns x nr values, r fastest (the Fortran (nr, ns, ncomp)
slab written column-major through MPI-IO with the single-precision type).

* ``Uface`` (9): block 1's fields at its q-max face, ``Vface`` (9): block
  2's at its q-min face, ``S`` (4): slip and its magnitude integral,
  ``state`` (1): the state variable -- all at t_(n-1), before the step;
* ``Uhat`` / ``Vhat`` (6): hat velocities (overwritten with v_hat - u_hat)
  and hat tractions plus prestress, ``Svel`` (3): the slip velocity (Uhat's
  first three components), ``trup`` (1): rupture time -- from stage 1 of step n.

:class:`FaultOutput` writes them from a :class:`Domain`;
:func:`run_with_fault_output` is time_step_RK's loop with write_output.
The files read back with the reference's python/read_binary.py layout:
``np.fromfile(f, np.float32).reshape(nt, ncomp, ns, nr)``.
"""
from __future__ import annotations

import numpy as np

FILES = (("Uface", 9), ("Vface", 9), ("S", 4), ("Uhat", 6), ("Vhat", 6), ("Svel", 3), ("trup", 1), ("state", 1))


class FaultOutput:
    """The eight ``<prefix>_interface.*`` files of one two-block run."""

    def __init__(self, domain, prefix: str):
        if domain.nblocks != 2:
            raise ValueError("fault output needs a two-block domain")
        self.domain = domain
        self.files = {name: open(f"{prefix}_interface.{name}", "wb") for name, _ in FILES}

    def _put(self, name: str, a: np.ndarray):
        np.ascontiguousarray(a, dtype=np.float32).tofile(self.files[name])

    def write_fault(self):
        """write_fault + the Vface write of write_fault_output (state before the step)."""
        d = self.domain
        # the two interface faces through the device plane gather
        self._put("Uface", d.plane(0, 1, d.blocks[0].nqrs[0]))
        self._put("Vface", d.plane(1, 1, 1))
        self._put("S", d.fault("S"))
        self._put("state", d.fault("state"))

    def write_hats(self):
        """write_hats (the stage-1 hat variables of the step just taken)."""
        d = self.domain
        self._put("Uhat", d.fault("Uhat"))
        self._put("Vhat", d.fault("Vhat"))
        self._put("Svel", d.fault("Svel"))
        self._put("trup", d.fault("trup"))

    def close(self):
        for f in self.files.values():
            f.close()
        self.files = {}

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def run_with_fault_output(domain, nsteps: int, prefix: str, first: int = 1) -> int:
    """Steps first .. first + nsteps - 1 one at a time with the reference's
    fault output at every w_stride-th step; returns the number of records."""
    w = max(int(domain.problem.w_stride), 1)
    nrec = 0
    with FaultOutput(domain, prefix) as fo:
        for n in range(first, first + nsteps):
            out = (n - 1) % w == 0
            if out:
                fo.write_fault()
            domain.time_step_RK(n)
            if out:
                fo.write_hats()
                nrec += 1
    return nrec


def read_fault_output(prefix: str, name: str, ns: int, nr: int) -> np.ndarray:
    """One file back as (nt, ncomp, ns, nr) float32, as python/read_binary.py reads it."""
    nc = dict(FILES)[name]
    a = np.fromfile(f"{prefix}_interface.{name}", dtype=np.float32)
    return a.reshape(-1, nc, ns, nr)
