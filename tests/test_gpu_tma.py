"""The Cartesian interior tile's planes filled by TMA box loads
(cp.async.bulk.tensor completing on an mbarrier per plane buffer,
WQL3D_TMA=1) against the same tile filled by per-thread 16-byte cp.async (the
default, WQL3D_TMA=0).  The staged values the stencil reads are the same, so
fields, memory variables and stations must agree bit for bit; the small
blocks put the last tile's box past the end of the padded rows (zero fill
outside the array).  The tuning switch is read once per process, so each
variant runs in a subprocess."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.abspath(__file__))

RUNNER = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[4])
from cases import small_case
from waveqlab3d_q_gpu_b200.domain import Domain
response, prec, out = sys.argv[1], sys.argv[2], sys.argv[3]
p = small_case(mesh="cartesian", response=response, n=(45, 31, 29))
g = Domain(p, precision=prec, nsteps_hint=12)
g.run(11)
ok = g.check_status()
res = {"F": g.fields(0), "S": g.seismograms(0)}
if response != "elastic":
    res["E"] = g.eta(0)
np.savez(out, **res)
g.close()
"""


def _run(tmp_path, response, prec, tma):
    env = dict(os.environ)
    env["WQL3D_TMA"] = str(tma)
    env["PYTHONPATH"] = os.path.dirname(ROOT) + os.pathsep + env.get("PYTHONPATH", "")
    out = str(tmp_path / f"{response}_{prec}_{tma}.npz")
    r = subprocess.run([sys.executable, "-c", RUNNER, response, prec, out, ROOT], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return np.load(out)


@pytest.mark.parametrize("response,prec", [("elastic", "fp64"), ("anelastic-Q8", "fp64"),
                                           ("anelastic-fQ8", "fp32"), ("anelastic-Q4", "fp32")])
def test_tma_planes_equal_cp_async_planes(wql3d_lib, tmp_path, response, prec):
    a = _run(tmp_path, response, prec, 0)
    b = _run(tmp_path, response, prec, 1)
    assert set(a.files) == set(b.files)
    for k in a.files:
        assert np.array_equal(a[k], b[k]), (k, np.abs(a[k] - b[k]).max())
    assert np.abs(a["F"]).max() > 0.0


STALL = r"""
import sys
sys.path.insert(0, sys.argv[1])
from cases import small_case
from waveqlab3d_q_gpu_b200.domain import Domain
from waveqlab3d_q_gpu_b200._lib import Wql3dError
p = small_case(mesh="cartesian", response="elastic", n=(45, 31, 29))
g = Domain(p, nsteps_hint=2)
g.time_step_RK()
try:
    g.check_status()
    print("NO-STALL")
except Wql3dError as e:
    print("STALL", e)
F = g.fields(0)
print("READ", F.shape)
g.close()
"""


def test_tma_wait_limit_reports_stall(wql3d_lib):
    """WQL3D_TMA=2 issues no copies: every plane wait runs out (bounded, about a
    second per tile), the tile carries on, the domain status reports the stall
    and the context stays usable."""
    env = dict(os.environ)
    env["WQL3D_TMA"] = "2"
    env["PYTHONPATH"] = os.path.dirname(ROOT) + os.pathsep + env.get("PYTHONPATH", "")
    r = subprocess.run([sys.executable, "-c", STALL, ROOT], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    assert "STALL" in r.stdout and "bounded wait" in r.stdout, r.stdout
    assert "READ (9, 29, 31, 45)" in r.stdout, r.stdout
