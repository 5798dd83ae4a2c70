"""Curvilinear block meshes by transfinite interpolation (Curve_Grid_3D3,
src/grid.f90:473-1909): the six boundary surfaces of the rupture test
profile, the oracle's volume interpolation (Gen3_Curve_Mesh,
src/grid.f90:2292-2418) reproducing them, and the device kernel against the
oracle."""
import numpy as np
import pytest

from waveqlab3d_q_gpu_b200.mesh import block_surfaces, pack_surfaces

CASES = [("flat", 0.0, 0.0), ("analytical_test_problem", 1.0, 0.0), ("analytical_test_problem", 0.0, 1.0)]


@pytest.mark.parametrize("profile,lc,rc", CASES)
def test_oracle_tfi_reproduces_the_surfaces(oracle_lib, profile, lc, rc):
    n = (21, 23, 25)
    s = block_surfaces(n, (-3.0, 6.0, -1.5), (0.0, 9.0, 1.5), lc, rc, profile)
    X = oracle_lib.tfi_grid(pack_surfaces(s), n)
    tol = 1e-14
    assert np.abs(X[:, :, :, 0] - s["left"]).max() < tol and np.abs(X[:, :, :, -1] - s["right"]).max() < tol
    assert np.abs(X[:, :, 0, :] - s["top"]).max() < tol and np.abs(X[:, :, -1, :] - s["bottom"]).max() < tol
    assert np.abs(X[:, 0] - s["front"]).max() < tol and np.abs(X[:, -1] - s["back"]).max() < tol
    if profile == "flat":
        q = np.linspace(-3.0, 0.0, n[0])
        assert np.abs(X[0] - q[None, None, :]).max() < 1e-14
    else:
        face = X[0, :, :, -1] if lc else X[0, :, :, 0]
        assert abs(np.abs(face - (0.0 if lc else -3.0)).max() - 0.1) < 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("profile,lc,rc", CASES)
def test_device_tfi_matches_oracle(wql3d_lib, oracle_lib, profile, lc, rc):
    from waveqlab3d_q_gpu_b200.mesh import tfi_grid
    n = (21, 23, 25)
    s = block_surfaces(n, (0.0, 6.0, -1.5), (3.0, 9.0, 1.5), lc, rc, profile)
    Xg = tfi_grid(s, n)
    Xo = oracle_lib.tfi_grid(pack_surfaces(s), n)
    assert np.abs(Xg - Xo).max() <= 1e-14 * np.abs(Xo).max()
