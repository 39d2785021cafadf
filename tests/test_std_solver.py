"""Host-side set-up of the single-species driver (no GPU needed)."""
import numpy as np
import pytest

from dgfs1d_gpu_b200.config import Config
from dgfs1d_gpu_b200.configs import couette_std_ini
from dgfs1d_gpu_b200.plugins import subclass_where
from dgfs1d_gpu_b200.velocitymesh import DGFSVelocityMeshStd


def test_couette_ini_knudsen_and_mesh():
    cfg = Config(couette_std_ini())
    vm = DGFSVelocityMeshStd(cfg)
    assert vm.L() == 5.0 and vm.Nv() == 16 and vm.M() == 6
    assert vm.sphere_mode() == 'half' and vm.sw() == 2 * np.pi / 6
    invKn = vm.H0() * np.sqrt(2.0) * np.pi * vm.n0() * 4.17e-10 ** 2
    assert abs(invKn - 10.0) < 1e-9


def test_full_sphere_when_no_half_rule():
    cfg = Config(couette_std_ini(Nv=32, M=12, Nrho=16, dev=6.0))
    vm = DGFSVelocityMeshStd(cfg)
    assert vm.sphere_mode() == 'full' and vm.sphere_factor() == 1.0
    assert vm.sz().shape == (12, 3)


def test_plugin_keys():
    from dgfs1d_gpu_b200.std import integrator, scattering  # noqa: F401
    from dgfs1d_gpu_b200.std.integrator import DGFSIntegratorStd
    from dgfs1d_gpu_b200.std.scattering import DGFSScatteringModelStd
    for k in ('euler', 'ssp-rk2', 'ssp-rk3', 'lse-rk45', 'lserk-45'):
        assert subclass_where(DGFSIntegratorStd, intg_kind=k)
    for k in ('vhs-gll', 'vhs'):
        assert subclass_where(DGFSScatteringModelStd, scattering_model=k)
    with pytest.raises(KeyError):
        subclass_where(DGFSIntegratorStd, intg_kind='rk4')
