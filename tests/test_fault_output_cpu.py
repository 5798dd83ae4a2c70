"""Fault output files (host side, no GPU): record layout, order of the
before-step and stage-1 writes, and the w_stride sampling, with a stand-in
domain whose outputs encode the step they were taken at."""
import numpy as np

from waveqlab3d_q_gpu_b200.fault_output import FILES, read_fault_output, run_with_fault_output


class _P:
    w_stride = 2


class _FakeDomain:
    nblocks = 2
    problem = _P()

    def __init__(self, ns=5, nr=7, nq=4):
        self.ns, self.nr, self.nq = ns, nr, nq
        self.step = 0

    def _grid(self, nc, tag):
        c = np.arange(nc)[:, None, None]
        s = np.arange(self.ns)[None, :, None]
        r = np.arange(self.nr)[None, None, :]
        return tag + 100.0 * c + 10.0 * s + r + 0.0 * (c + s + r)

    def fields(self, b):
        F = np.zeros((9, self.ns, self.nr, self.nq))
        F[:, :, :, -1 if b == 0 else 0] = self._grid(9, 1000.0 * self.step + b)
        return F

    def fault(self, name):
        return self._grid(dict(FILES)[name], 1000.0 * self.step + 0.5)

    @property
    def blocks(self):
        from types import SimpleNamespace
        return [SimpleNamespace(nqrs=(self.nq, self.nr, self.ns))] * 2

    def plane(self, b, axis, index, c0=0, ncomp=9):
        # the device plane gather of Domain.plane, on the fake fields
        assert axis == 1
        return self.fields(b)[c0:c0 + ncomp, :, :, index - 1]

    def time_step_RK(self, n):
        self.step = n


def test_layout_order_and_stride(tmp_path):
    d = _FakeDomain()
    prefix = str(tmp_path / "run")
    assert run_with_fault_output(d, 5, prefix) == 3          # steps 1, 3, 5
    for name, nc in FILES:
        a = read_fault_output(prefix, name, d.ns, d.nr)
        assert a.shape == (3, nc, d.ns, d.nr)
        # before-step files hold step n-1's values, the hat files step n's
        before = name in ("Uface", "Vface", "S", "state")
        for i, n in enumerate((1, 3, 5)):
            tag = 1000.0 * (n - 1 if before else n) + (1 if name == "Vface" else 0 if name == "Uface" else 0.5)
            assert np.array_equal(a[i], d._grid(nc, tag).astype(np.float32)), (name, i)
