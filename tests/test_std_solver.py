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


def test_astd_plugin_keys():
    """Every IMEX scheme and penalty model key of the reference's
    dgfsABstd1D that this package implements resolves."""
    from dgfs1d_gpu_b200.astd.integrator import DGFSIntegratorAstd
    from dgfs1d_gpu_b200.astd.scattering import DGFSScatteringModelAstd
    for k in ('bdf-111', 'bdf-222', 'imex-lm-bdf1', 'imex-lm-bdf2',
              'imex-lm-cn2', 'imex-lm-ad2', 'imex-lm-sg2', 'imex-lm-bdf3',
              'imex-lm-ad3', 'imex-lm-tvb3', 'imex-lm-bdf4', 'imex-lm-tvb4',
              'imex-lm-shu3', 'imex-lm-shu4'):
        cls = subclass_where(DGFSIntegratorAstd, intg_kind=k)
        if k.startswith('imex-lm'):
            assert len(cls.B) == len(cls.A) and len(cls.C) == len(cls.A) + 1
    for k, na in (('bgk-direct-gll', 5), ('boltz-bgk-direct-gll', 5),
                  ('esbgk-direct-gll', 11), ('boltz-esbgk-direct-gll', 11),
                  ('shakov-direct-gll', 14), ('boltz-shakov-direct-gll', 14)):
        assert subclass_where(DGFSScatteringModelAstd, scattering_model=k).nalph == na


def test_sod_shock_tube_initial_condition():
    """sod-shock-tube (std/initcond.py:320-383): left elements hold the left
    Maxwellian, right elements the right one (dimensional inputs)."""
    from dgfs1d_gpu_b200.std.initcond import get_initcond
    ini = couette_std_ini(Nv=16, Ne=4) + """
[soln-ics]
type = sod-shock-tube
rho-left = 2.0e-4
T-left = 300
rho-right = 1.0e-4
T-right = 250
"""
    cfg = Config(ini.replace('[soln-ics]\ntype = maxwellian', '[ignored-ics]\ntype = maxwellian', 1))
    vm = DGFSVelocityMeshStd(cfg)
    usol = np.zeros((3, 4, vm.vsize()))
    get_initcond(cfg, vm, 'soln-ics').apply_init_vals(usol, 3, 4, None)
    cv = vm.cv()
    for e, (rho, T) in enumerate([(2.0e-4, 300), (2.0e-4, 300), (1.0e-4, 250), (1.0e-4, 250)]):
        r, t = rho / vm.rho0(), T / vm.T0()
        M = r / (np.pi * t) ** 1.5 * np.exp(-np.sum(cv ** 2, axis=0) / t)
        assert np.allclose(usol[:, e, :], M[None, :], rtol=1e-14, atol=0)
