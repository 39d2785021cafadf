"""Mixture initial conditions (``[soln-ics] type``), dgfs1D/bi/initcond.py.

``maxwellian``: species p gets nden_p (m_p/(pi T))^{3/2} exp(-m_p|c-u|^2/T)
with nden_p = nden{p+1}/n0 (wall=True: nden_p = 1).  ``maxwellian-noise``
(new) multiplies by (1 + amp U[-1, 1]) i.i.d. per phase-space point.
"""
import numpy as np

from ..plugins import subclass_where


class DGFSInitConditionBi:
    model = None

    def __init__(self, cfg, vm, name, **kwargs):
        self.cfg, self.vm, self.name = cfg, vm, name
        self._nspcs = vm.nspcs()
        self.load_parameters(name, **kwargs)
        self.perform_precomputation()

    def get_init_vals(self):
        return self._init_vals

    def apply_init_vals(self, p, usol, Nq, Ne, xsol=None):
        usol[:, :, :] = self._init_vals[p][None, None, :]


class DGFSMaxwellianInitConditionBi(DGFSInitConditionBi):
    model = 'maxwellian'

    def load_parameters(self, name, wall=False):
        vm, cfg = self.vm, self.cfg
        u0 = vm.u0()
        self._nden = [1.0] * self._nspcs
        if not wall:
            self._nden = [cfg.lookupfloat(name, 'nden%d' % (i + 1)) / vm.n0()
                          for i in range(self._nspcs)]
        self._Tini = cfg.lookupfloat(name, 'T') / vm.T0()
        self._uini = np.array([cfg.lookupfloat(name, 'ux') / u0,
                               cfg.lookupfloat(name, 'uy') / u0,
                               cfg.lookupfloat(name, 'uz') / u0]).reshape(3, 1)

    def perform_precomputation(self):
        m = self.vm.masses()
        cv = self.vm.cv()
        self._init_vals = [
            self._nden[p] * ((m[p] / np.pi / self._Tini) ** 1.5)
            * np.exp(-m[p] * np.sum((cv - self._uini) ** 2, axis=0) / self._Tini)
            for p in range(self._nspcs)]

    def unondim(self):
        return self._uini


class DGFSMaxwellianNoiseInitConditionBi(DGFSMaxwellianInitConditionBi):
    model = 'maxwellian-noise'

    def load_parameters(self, name, wall=False):
        super().load_parameters(name, wall)
        self._amp = self.cfg.lookupordefault(name, 'noise', 0.01)
        self._seed = self.cfg.lookupordefault(name, 'seed', 20261203)

    def apply_init_vals(self, p, usol, Nq, Ne, xsol=None):
        rng = np.random.default_rng(self._seed + p)
        usol[:, :, :] = self._init_vals[p][None, None, :] * (
            1 + self._amp * rng.uniform(-1, 1, usol.shape))


def get_initcond(cfg, vm, name, **kwargs):
    cls = subclass_where(DGFSInitConditionBi, model=cfg.lookup(name, 'type'))
    return cls(cfg, vm, name, **kwargs)
