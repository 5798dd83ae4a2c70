"""Plane and slice writers on the CUDA path: the device plane gather
(wql3d_get_plane) against the full field readback, the .plane files of
src/plane_output.f90 read back header and records, and the .Hslice / .Vslice
files of a GPU TPV5 run against the oracle's planes and the archived slices
(test_problems/truth/1, the cores that test_oracle_slices.py pins)."""
import os

import numpy as np
import pytest

from cases import small_case, tpv5_case

pytestmark = pytest.mark.gpu


def _domain(problem, **kw):
    from waveqlab3d_q_gpu_b200.domain import Domain
    return Domain(problem, **kw)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_plane_gather_equals_field_readback(wql3d_lib, precision):
    p = small_case(mesh="curvilinear", response="elastic")
    g = _domain(p, precision=precision, nsteps_hint=5)
    g.run(5)
    F = g.fields(0)                                  # (9, ns, nr, nq)
    nq, nr, ns = p.blocks[0].nqrs
    for axis, n in ((1, nq), (2, nr), (3, ns)):
        for index in (1, n // 2, n):
            for c0, nc in ((0, 9), (0, 3), (4, 2)):
                a = g.plane(0, axis, index, c0, nc)
                if axis == 1:
                    ref = F[c0:c0 + nc, :, :, index - 1]
                elif axis == 2:
                    ref = F[c0:c0 + nc, :, index - 1, :]
                else:
                    ref = F[c0:c0 + nc, index - 1, :, :]
                assert np.array_equal(a, ref), (axis, index, c0, nc)
    from waveqlab3d_q_gpu_b200._lib import Wql3dError
    for bad in ((4, 1, 0, 9), (1, nq + 1, 0, 9), (1, 0, 0, 9), (1, 1, 8, 2)):
        with pytest.raises(Wql3dError):
            g.plane(0, *bad)
    g.close()


def test_plane_files(wql3d_lib, tmp_path):
    from waveqlab3d_q_gpu_b200.plane_output import PlaneOutput, read_plane
    p = tpv5_case()
    g = _domain(p, nsteps_hint=6)
    out = PlaneOutput(g, ["yz", "xy", "qr", "xz"], [-1.5, 0.3, 5.0, 99.0], names=["x", "z", "k5", "off"], stride=2,
                      directory=str(tmp_path), domain_name="tpv5")
    recs = {}
    for n in range(1, 7):
        for pl in out.planes:
            if pl.active and (pl.counter % pl.stride) == 0:
                recs.setdefault(pl.path, []).append((g.t, g.fields(pl.block)[0:3].copy()))
        out.write()
        g.time_step_RK(n)
    out.close()
    names = sorted(os.listdir(tmp_path))
    # 'yz' at x = -1.5 lies in block 1 only, 'off' (y = 99) in neither block
    assert "tpv5_x_block1.plane" in names and "tpv5_x_block2.plane" not in names
    assert not any("off" in f for f in names)
    for pl in out.planes:
        if not pl.active:
            continue
        hdr, t, v = read_plane(pl.path)
        assert hdr["version"] == 1 and hdr["axis"] == pl.axis_id and hdr["index"] == pl.index
        assert (hdr["n1"], hdr["n2"]) == (pl.n1, pl.n2) and hdr["coord"] == pl.coord
        assert len(t) == 3                     # stride 2 over 6 calls
        for k, (tk, F) in enumerate(recs[pl.path]):
            assert t[k] == tk
            if pl.fdir == 1:
                ref = F[:, :, :, pl.index - 1]
            elif pl.fdir == 2:
                ref = F[:, :, pl.index - 1, :]
            else:
                ref = F[:, pl.index - 1, :, :]
            assert np.array_equal(v[k], ref)
    g.close()


def test_slice_files_match_oracle_and_archive(wql3d_lib, oracle_lib, tmp_path):
    from waveqlab3d_q_gpu_b200.plane_output import SliceOutput, read_slice
    golden = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rupture_slices.npz"))
    p = tpv5_case()
    g = _domain(p, nsteps_hint=4)
    o = oracle_lib.OracleDomain(p)
    name = str(tmp_path / "test_rup_cart_fric")
    oh, ov = [], []
    with SliceOutput(g, name, horz=True, vert=True) as so:
        for n in range(1, 5):
            so.write()
            F = o.fields(0)
            oh.append(F[:, :, 0, :])
            ov.append(F[:, 0, :, :])
            g.time_step_RK(n)
            o.run(1)
    H = read_slice(name + ".Hslice", 21, 21)
    V = read_slice(name + ".Vslice", 21, 21)
    assert os.path.getsize(name + ".Hslice") == 4 * 9 * 21 * 21 * 4
    for k in range(4):
        for mine, ref, arch in ((H[k], oh[k], golden["tpv5_H"][k]), (V[k], ov[k], golden["tpv5_V"][k])):
            scale = max(np.abs(ref).max(), 1e-30)
            assert np.abs(mine - ref).max() <= 1e-6 * scale + 1e-37
            if k:
                assert np.abs(mine - arch)[:, :, :14].max() / np.abs(arch).max() < (5e-6 if k == 1 else 1e-4)
    g.close()
