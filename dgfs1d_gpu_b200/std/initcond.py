"""Initial-condition plugins (``[soln-ics] type``) of the single-species solver.

``maxwellian`` and ``bkw`` restate dgfs1D/std/initcond.py:36-141 (values on
the velocity grid, nondimensional).  ``maxwellian-noise`` (no counterpart in
the reference) multiplies the Maxwellian by (1 + amp U[-1, 1]), i.i.d. per
phase-space point from a seeded generator (keys ``noise``, ``seed``).
"""
import numpy as np

from ..plugins import subclass_where


class DGFSInitConditionStd:
    model = None

    def __init__(self, cfg, vm, name, **kwargs):
        self.cfg, self.vm, self.name = cfg, vm, name
        self.load_parameters(name, **kwargs)
        self.perform_precomputation()

    def get_init_vals(self):
        return self._init_vals

    def apply_init_vals(self, usol, Nq, Ne, xsol=None):
        usol[:, :, :] = self._init_vals[None, None, :]


class DGFSMaxwellianInitConditionStd(DGFSInitConditionStd):
    model = 'maxwellian'

    def load_parameters(self, name, wall=False):
        vm, cfg = self.vm, self.cfg
        u0 = vm.u0()
        self._rhoini = 1.0
        if not wall:
            self._rhoini = cfg.lookupfloat(name, 'rho') / vm.rho0()
        self._Tini = cfg.lookupfloat(name, 'T') / vm.T0()
        self._uini = np.array([cfg.lookupfloat(name, 'ux') / u0,
                               cfg.lookupfloat(name, 'uy') / u0,
                               cfg.lookupfloat(name, 'uz') / u0]).reshape(3, 1)

    def perform_precomputation(self):
        self._init_vals = ((self._rhoini / (np.pi * self._Tini) ** 1.5)
                           * np.exp(-np.sum((self.vm.cv() - self._uini) ** 2,
                                            axis=0) / self._Tini))

    def unondim(self):
        return self._uini


class DGFSMaxwellianNoiseInitConditionStd(DGFSMaxwellianInitConditionStd):
    model = 'maxwellian-noise'

    def load_parameters(self, name, wall=False):
        super().load_parameters(name, wall)
        self._amp = self.cfg.lookupordefault(name, 'noise', 0.01)
        self._seed = self.cfg.lookupordefault(name, 'seed', 20261203)

    def apply_init_vals(self, usol, Nq, Ne, xsol=None):
        rng = np.random.default_rng(self._seed)
        usol[:, :, :] = self._init_vals[None, None, :] * (
            1 + self._amp * rng.uniform(-1, 1, usol.shape))


class DGFSBKWInitConditionStd(DGFSInitConditionStd):
    model = 'bkw'

    def load_parameters(self, name):
        self._t0 = self.cfg.lookupfloat(name, 't0')

    def perform_precomputation(self):
        K = 1.0 - np.exp(-self._t0 / 6.0)
        cSqr = np.sum(self.vm.cv() ** 2, axis=0)
        self._init_vals = (1 / (2 * pow(2 * np.pi * K, 1.5))
                           * np.exp(-cSqr / (2.0 * K))
                           * ((5 * K - 3) / K + (1 - K) / (K * K) * cSqr))


def get_initcond(cfg, vm, name, **kwargs):
    cls = subclass_where(DGFSInitConditionStd, model=cfg.lookup(name, 'type'))
    return cls(cfg, vm, name, **kwargs)
