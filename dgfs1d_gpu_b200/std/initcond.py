"""Initial-condition plugins (``[soln-ics] type``) of the single-species solver.

``maxwellian``, ``bkw`` and ``sod-shock-tube`` restate dgfs1D/std/
initcond.py:36-141, 320-383 (values on the velocity grid, nondimensional).  ``maxwellian-noise`` (no counterpart in
the reference) multiplies the Maxwellian by (1 + amp U[-1, 1]), i.i.d. per
phase-space point from a seeded generator (keys ``noise``, ``seed``).
``maxwellian-expr`` / ``maxwellian-expr-nondim`` and ``sod-shock-tube-nondim``
(initcond.py:144-238, 282-300, 385-434) evaluate their keys as expressions
of the nondimensional solution-point coordinate ``x`` and the values of the
``[non-dim]`` and ``[mesh]`` sections; the two Maxwellian-expression models
also take the optional ``noise``/``seed`` keys of ``maxwellian-noise`` (no
counterpart in the reference).
``normal-shock`` (no counterpart in the reference) joins an upstream and a
downstream Maxwellian by a tanh ramp in x (keys ``rho1 T1 ux1 rho2 T2 ux2``,
dimensional like ``maxwellian``; ``x0``, ``width`` in mesh units; optional
``noise``, ``seed``).
"""
import numpy as np

from ..config import npeval
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


class DGFSNormalShockInitConditionStd(DGFSInitConditionStd):
    model = 'normal-shock'

    def load_parameters(self, name):
        vm, cfg = self.vm, self.cfg
        u0 = vm.u0()
        self._states = []
        for k in ('1', '2'):
            rho = cfg.lookupfloat(name, 'rho' + k) / vm.rho0()
            T = cfg.lookupfloat(name, 'T' + k) / vm.T0()
            ux = cfg.lookupfloat(name, 'ux' + k) / u0
            self._states.append((rho, T, ux))
        self._x0 = cfg.lookupfloat(name, 'x0') / vm.H0()
        self._w = cfg.lookupfloat(name, 'width') / vm.H0()
        self._amp = cfg.lookupordefault(name, 'noise', 0.0)
        self._seed = cfg.lookupordefault(name, 'seed', 20261203)

    def perform_precomputation(self):
        cv = self.vm.cv()
        self._M = []
        for rho, T, ux in self._states:
            u = np.array([ux, 0.0, 0.0]).reshape(3, 1)
            self._M.append(rho / (np.pi * T) ** 1.5
                           * np.exp(-np.sum((cv - u) ** 2, axis=0) / T))
        self._init_vals = self._M[0]

    def apply_init_vals(self, usol, Nq, Ne, xsol=None):
        w = 0.5 * (1 + np.tanh((np.asarray(xsol) - self._x0) / self._w))
        usol[:, :, :] = ((1 - w)[:, :, None] * self._M[0][None, None, :]
                         + w[:, :, None] * self._M[1][None, None, :])
        if self._amp:
            rng = np.random.default_rng(self._seed)
            usol *= 1 + self._amp * rng.uniform(-1, 1, usol.shape)


class DGFSSodShockTubeInitConditionStd(DGFSInitConditionStd):
    """Sod shock tube (std/initcond.py:320-383): the left half of the
    elements holds the Maxwellian (rho-left, T-left, ux-left), the right half
    (rho-right, T-right, ux-right), dimensional as ``maxwellian``; Ne must be
    even, and each Maxwellian's density must be resolved by the grid."""
    model = 'sod-shock-tube'

    def load_parameters(self, name):
        vm, cfg = self.vm, self.cfg
        self._states = []
        for side in ('left', 'right'):
            rho = cfg.lookupfloat(name, 'rho-' + side) / vm.rho0()
            T = cfg.lookupfloat(name, 'T-' + side) / vm.T0()
            ux = cfg.lookupordefault(name, 'ux-' + side, 0.) / vm.u0()
            self._states.append((rho, T, ux))

    def perform_precomputation(self):
        cv, cw = self.vm.cv(), self.vm.cw()
        self._M = []
        for rho, T, ux in self._states:
            u = np.array([ux, 0.0, 0.0]).reshape(3, 1)
            M = rho / (np.pi * T) ** 1.5 * np.exp(-np.sum((cv - u) ** 2, axis=0) / T)
            if not np.allclose(rho, np.sum(M) * cw, atol=1e-5):
                raise ValueError('Bulk properties not conserved! Check Nv, dev')
            self._M.append(M)
        self._init_vals = self._M[0]

    def get_init_vals(self):
        raise ValueError('this model depends on spatial coordinates!')

    def unondim(self):
        raise ValueError('this model depends on spatial coordinates!')

    def apply_init_vals(self, usol, Nq, Ne, xsol=None):
        if Ne % 2:
            raise ValueError('Not implemented')
        usol[:, :Ne // 2, :] = self._M[0][None, None, :]
        usol[:, Ne // 2:, :] = self._M[1][None, None, :]


def _maxwellian(cv, rho, ux, uy, uz, T):
    """rho / (pi T)^1.5 exp(-|c - u|^2 / T) for every point of the (...,)
    shaped state arrays, on the velocity grid cv (3, Nv): shape (..., Nv)."""
    rho, ux, uy, uz, T = np.broadcast_arrays(*[np.asarray(a, dtype=np.float64)
                                              for a in (rho, ux, uy, uz, T)])
    out = np.empty(rho.shape + (cv.shape[1],))
    flat = out.reshape(-1, cv.shape[1])
    for i, (r, a, b, c, t) in enumerate(zip(rho.ravel(), ux.ravel(), uy.ravel(),
                                            uz.ravel(), T.ravel())):
        c2 = (cv[0] - a) ** 2 + (cv[1] - b) ** 2 + (cv[2] - c) ** 2
        flat[i] = r / (np.pi * t) ** 1.5 * np.exp(-c2 / t)
    return out


def _expr_vars(cfg, xsol):
    v = {}
    v.update(cfg.section_values('non-dim', np.float64))
    v.update(cfg.section_values('mesh', np.float64))
    v['x'] = xsol
    return v


class DGFSMaxwellianExprInitConditionStd(DGFSInitConditionStd):
    """Maxwellian whose rho, ux, uy, uz, T are expressions of x
    (initcond.py:144-238), dimensional (scaled by rho0, u0, T0)."""
    model = 'maxwellian-expr'
    _scaled = True

    def load_parameters(self, name):
        self._exprs = {k: self.cfg.lookupexpr(name, k)
                       for k in ('rho', 'ux', 'uy', 'uz', 'T')}
        self._amp = float(self.cfg.lookupordefault(name, 'noise', 0.0))
        self._seed = int(self.cfg.lookupordefault(name, 'seed', 20261203))

    def perform_precomputation(self):
        pass

    def get_init_vals(self):
        raise ValueError('this model depends on spatial coordinates!')

    def unondim(self):
        raise ValueError('this model depends on spatial coordinates!')

    def states(self, xsol):
        vm = self.vm
        v = _expr_vars(self.cfg, xsol)
        sc = dict(rho=vm.rho0(), ux=vm.u0(), uy=vm.u0(), uz=vm.u0(), T=vm.T0())
        out = {}
        for k, e in self._exprs.items():
            val = np.asarray(npeval(e, v), dtype=np.float64)
            out[k] = val / sc[k] if self._scaled else val
        return out

    def apply_init_vals(self, usol, Nq, Ne, xsol=None):
        st = self.states(xsol)
        shape = (Nq, Ne)
        st = {k: np.broadcast_to(v, shape) for k, v in st.items()}
        usol[...] = _maxwellian(self.vm.cv(), st['rho'], st['ux'], st['uy'],
                                st['uz'], st['T'])
        if self._amp:
            rng = np.random.default_rng(self._seed)
            usol *= 1 + self._amp * rng.uniform(-1, 1, usol.shape)


class DGFSMaxwellianExprNonDimInitConditionStd(
        DGFSMaxwellianExprInitConditionStd):
    """``maxwellian-expr`` with nondimensional values (initcond.py:282-300)."""
    model = 'maxwellian-expr-nondim'
    _scaled = False


class DGFSSodShockNonDimTubeInitConditionStd(DGFSInitConditionStd):
    """Nondimensional Sod tube (initcond.py:385-434): rho-, T-, ux-left/right
    are expressions of x; points with x <= xMid take the left state; every
    Maxwellian's density must be resolved by the grid (atol 1e-5)."""
    model = 'sod-shock-tube-nondim'

    def load_parameters(self, name):
        cfg = self.cfg
        self._exprs = {'%s-%s' % (k, s): cfg.lookupexpr(name, '%s-%s' % (k, s))
                       for k in ('rho', 'T', 'ux') for s in ('left', 'right')}
        self._xmid = cfg.lookupfloat(name, 'xMid')

    def perform_precomputation(self):
        pass

    def get_init_vals(self):
        raise ValueError('this model depends on spatial coordinates!')

    def unondim(self):
        raise ValueError('this model depends on spatial coordinates!')

    def apply_init_vals(self, usol, Nq, Ne, xsol=None):
        v = _expr_vars(self.cfg, xsol)
        val = {k: np.broadcast_to(np.asarray(npeval(e, v), dtype=np.float64),
                                  (Nq, Ne)).ravel()
               for k, e in self._exprs.items()}
        x = np.asarray(xsol).ravel()
        flat = usol.reshape(-1, usol.shape[-1])
        cv, cw = self.vm.cv(), self.vm.cw()
        for side, sel in (('left', x <= self._xmid), ('right', x > self._xmid)):
            rho = val['rho-' + side][sel]
            M = _maxwellian(cv, rho, val['ux-' + side][sel], 0.0, 0.0,
                            val['T-' + side][sel])
            if not np.allclose(rho, M.sum(axis=-1) * cw, atol=1e-5):
                raise ValueError('Bulk properties not conserved! Check Nv, dev')
            flat[sel, :] = M
