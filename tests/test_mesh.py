"""Host-side setup: package meshes and rules agree with the oracle."""
import numpy as np
import pytest

from dgfs1d_gpu_b200.quadrature import gauss_jacobi, gauss_lobatto_jacobi
from dgfs1d_gpu_b200.sphericaldesign import get_sphquadrule
from dgfs1d_gpu_b200.workloads import vhs_mesh_params
from oracle import mesh as om


@pytest.mark.parametrize('n', [2, 3, 4, 6, 8, 12, 16, 24])
def test_gauss_rules(n):
    z, w = gauss_jacobi(n)
    z0, w0 = om.gauss_jacobi(n)
    assert np.allclose(z, z0, atol=1e-14) and np.allclose(w, w0, atol=1e-14)
    # exactness for polynomials of degree 2n-1
    for k in range(2 * n):
        assert abs(w @ z ** k - (1 - (-1) ** (k + 1)) / (k + 1)) < 1e-12
    if n >= 2:
        zl, wl = gauss_lobatto_jacobi(n)
        zl0, wl0 = om.gauss_lobatto_jacobi(n)
        assert np.allclose(zl, zl0, atol=1e-14)
        assert np.allclose(wl, wl0, atol=1e-14)


@pytest.mark.parametrize('m', [6, 12, 32, 192])
def test_sphere_designs_antipodal(m):
    pts = get_sphquadrule('symmetric', 'womersley', npts=m).pts
    assert pts.shape == (m, 3)
    assert np.allclose(np.linalg.norm(pts, axis=1), 1, atol=1e-14)
    assert np.array_equal(pts[m // 2:], -pts[:m // 2])


@pytest.mark.parametrize('case', [(16, 6, 8, 5., False), (32, 12, 16, 6., True)])
def test_mesh_params_match_oracle(case):
    N, M, Nrho, dev, full = case
    prm = vhs_mesh_params(N, M, Nrho, dev, full)
    vm = om.VelocityMeshStd(Nv=N, M=M, Nrho=Nrho, dev=dev, full_sphere=full)
    _, prefac = om.vhs_prefactor(vm, 0.81, 4.17e-10, 273.)
    assert prm['L'] == vm.L and prm['cw'] == vm.cw
    assert np.allclose(prm['qz'], vm.qz, rtol=1e-15, atol=0)
    assert np.allclose(prm['qw'], vm.qw, rtol=1e-14, atol=0)
    assert np.array_equal(prm['sz'], vm.sz)
    assert prm['sw'] == vm.sw and prm['sphere_factor'] == vm.sphere_factor
    assert abs(prm['prefac'] / prefac - 1) < 1e-15
    assert np.array_equal(prm['c0'], vm.cv[2, :N])
