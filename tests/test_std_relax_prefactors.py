"""Prefactors of the explicit relaxation models of dgfsStd1D against the
reference's load_parameters formulas, restated here:
  bgk-direct-gll    t0 Pr p0 / visc with Pr = 1   (std/scattering.py:1196-1206)
  esbgk-direct-gll  t0 Pr p0 / visc, Pr from the config, default 2/3
                                                  (std/scattering.py:1382-1392)
  shakov-direct-gll t0 p0 / visc (Pr not applied)  (std/scattering.py:1648-1658)
with t0 = H0/u0, visc = muRef (T0/Tref)^omega, p0 = n0 R0/NA T0."""
import pytest

from dgfs1d_gpu_b200.config import Config
from dgfs1d_gpu_b200.configs import couette_std_ini
from dgfs1d_gpu_b200.plugins import subclass_where
from dgfs1d_gpu_b200.std.scattering import DGFSScatteringModelStd
from dgfs1d_gpu_b200.velocitymesh import DGFSVelocityMeshStd


def _reference_prefactor(cfg, vm, model):
    omega = cfg.lookupfloat('scattering-model', 'omega')
    muRef = cfg.lookupfloat('scattering-model', 'muRef')
    Tref = cfg.lookupfloat('scattering-model', 'Tref')
    Pr = float(cfg.lookupordefault('scattering-model', 'Pr', 2. / 3.))
    t0 = vm.H0() / vm.u0()
    visc = muRef * ((vm.T0() / Tref) ** omega)
    p0 = vm.n0() * vm.R0 / vm.NA * vm.T0()
    if model == 'bgk-direct-gll':
        return t0 * 1.0 * p0 / visc, 1.0
    if model == 'esbgk-direct-gll':
        return t0 * Pr * p0 / visc, Pr
    return t0 * p0 / visc, Pr


@pytest.mark.parametrize('Pr', [None, 0.71])
@pytest.mark.parametrize('model', ['bgk-direct-gll', 'esbgk-direct-gll',
                                   'shakov-direct-gll'])
def test_prefactor_matches_reference_formula(model, Pr):
    ini = couette_std_ini(Nv=8, Nrho=4).replace('type = vhs-gll',
                                                 'type = %s' % model)
    if Pr is not None:
        ini = ini.replace('[scattering-model]', '[scattering-model]\nPr = %r' % Pr)
    cfg = Config(ini)
    vm = DGFSVelocityMeshStd(cfg)
    cls = subclass_where(DGFSScatteringModelStd, scattering_model=model)
    sm = cls(cfg, vm, Ne=4)
    ref, ref_Pr = _reference_prefactor(cfg, vm, model)
    assert sm.prefac == pytest.approx(ref, rel=1e-14)
    assert sm._Pr == pytest.approx(ref_Pr, rel=1e-15)
