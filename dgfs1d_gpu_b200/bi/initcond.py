"""Mixture initial conditions (``[soln-ics] type``), dgfs1D/bi/initcond.py.

``maxwellian``: species p gets nden_p (m_p/(pi T))^{3/2} exp(-m_p|c-u|^2/T)
with nden_p = nden{p+1}/n0 (wall=True: nden_p = 1).  ``maxwellian-expr``
(:131-205): the same with nden{p+1}, ux, uy, uz, T expressions of the
solution-point coordinate x (dimensional), each Maxwellian's density
resolved by the grid (atol 1e-5).  ``maxwellian-noise`` (new) multiplies by
(1 + amp U[-1, 1]) i.i.d. per phase-space point.
"""
import numpy as np

from ..config import npeval
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


class DGFSMaxwellianExprInitConditionBi(DGFSInitConditionBi):
    model = 'maxwellian-expr'

    def load_parameters(self, name, **kwargs):
        pass

    def perform_precomputation(self):
        pass

    def get_init_vals(self):
        raise ValueError('this model depends on spatial coordinates!')

    def unondim(self):
        raise ValueError('this model depends on spatial coordinates!')

    def apply_init_vals(self, p, usol, Nq, Ne, xsol=None):
        if not 0 <= p < self._nspcs:
            raise ValueError('species index out of range')
        vm, cfg, name = self.vm, self.cfg, self.name
        m, cv, cw = vm.masses()[p], vm.cv(), vm.cw()
        v = {'x': xsol}
        ev = lambda k, s: np.broadcast_to(
            np.asarray(npeval(cfg.lookupexpr(name, k), v), dtype=np.float64) / s,
            (Nq, Ne))
        nden = ev('nden%d' % (p + 1), vm.n0())
        ux, uy, uz = (ev(k, vm.u0()) for k in ('ux', 'uy', 'uz'))
        T = ev('T', vm.T0())
        for q in range(Nq):
            for e in range(Ne):
                c2 = ((cv[0] - ux[q, e]) ** 2 + (cv[1] - uy[q, e]) ** 2
                      + (cv[2] - uz[q, e]) ** 2)
                f = nden[q, e] * ((m / np.pi / T[q, e]) ** 1.5) * np.exp(
                    -m * c2 / T[q, e])
                if not np.allclose(nden[q, e], np.sum(f) * cw, atol=1e-5):
                    raise ValueError('Bulk properties not conserved! Check Nv, dev')
                usol[q, e, :] = f


def get_initcond(cfg, vm, name, **kwargs):
    cls = subclass_where(DGFSInitConditionBi, model=cfg.lookup(name, 'type'))
    return cls(cfg, vm, name, **kwargs)
