"""Velocity meshes of the single-species and binary-mixture solvers (host).

Single species: dgfs1D/std/velocitymesh.py:8-129.  Binary mixture:
dgfs1D/bi/velocitymesh.py:7-144.  Same INI keys and the same derived
quantities: domain [-L, L]^3 with L = cmax/u0 + dev sqrt(Tmax/T0), N^3
cell-centred points, cell volume cw = (2L/N)^3, radial Gauss-Jacobi rule on
[0, R] and a spherical design.

Spherical rule (single species): the reference keeps the first M points of
the 2M-point symmetric design (a half sphere, weight 2 pi / M, factor 2 in
the gain sum).  When no 2M-point design exists (M = 12, 32, ...) the
full-sphere M-point design is used with weight 4 pi / M and factor 1 -- the
mixture convention -- selected by ``[spherical-design-rule] sphere = auto``
(default), or forced with ``half`` / ``full``.
"""
import numpy as np

from .quadrature import gauss_jacobi, gauss_lobatto_jacobi
from .sphericaldesign import available, get_sphquadrule

R0 = 8.3144598
NA = 6.0221409e+23


def _radial_rule(cfg, Nrho, R):
    kind = cfg.lookupordefault('velocity-mesh', 'quad-rule', 'jacobi')
    a = cfg.lookupordefault('velocity-mesh', 'quad-rule-alpha', 0.0)
    b = cfg.lookupordefault('velocity-mesh', 'quad-rule-beta', 0.0)
    rules = {'jacobi': gauss_jacobi, 'lobatto': gauss_lobatto_jacobi}
    if kind not in rules:
        raise ValueError('Valid quads: ' + str(list(rules)))
    z, w = rules[kind](Nrho, a, b)
    return (R / 2.0) * (1.0 + z), ((R - 0.0) / 2.0) * w


class _MeshBase:
    def _nondim(self, cfg):
        self._H0 = cfg.lookupfloat('mesh', 'H0')
        self._T0 = cfg.lookupfloat('non-dim', 'T0')
        self._rho0 = cfg.lookupfloat('non-dim', 'rho0')
        self._molarMass0 = cfg.lookupfloat('non-dim', 'molarMass0')
        self._n0 = self._rho0 / self._molarMass0 * NA
        self._u0 = np.sqrt(2 * R0 / self._molarMass0 * self._T0)
        self._Nv = cfg.lookupint('velocity-mesh', 'Nv')
        self._vsize = self._Nv ** 3
        self._Nrho = cfg.lookupordefault('velocity-mesh', 'Nrho',
                                         int(self._Nv / 2))
        cmax = cfg.lookupfloat('velocity-mesh', 'cmax') / self._u0
        Tmax = cfg.lookupfloat('velocity-mesh', 'Tmax') / self._T0
        self._dev = cfg.lookupfloat('velocity-mesh', 'dev')
        self._L = float(cmax + self._dev * np.sqrt(Tmax))
        return cmax, Tmax

    def _grid(self):
        N, L = self._Nv, self._L
        self._cw = (2.0 * L / N) ** 3
        self._c0 = np.linspace(-L + L / N, L - L / N, N)
        g = np.meshgrid(self._c0, self._c0, self._c0, indexing='ij')
        self._cv = np.stack([x.ravel() for x in g])

    def Nv(self): return self._Nv
    def Nrho(self): return self._Nrho
    def M(self): return self._M
    def L(self): return self._L
    def dev(self): return self._dev
    def vsize(self): return self._vsize
    def qz(self): return self._qz
    def qw(self): return self._qw
    def cv(self): return self._cv
    def c0(self): return self._c0
    def cw(self): return self._cw
    def sz(self): return self._sz
    def sw(self): return self._sw
    def sphere_factor(self): return self._sphere_factor
    def H0(self): return self._H0
    def T0(self): return self._T0
    def rho0(self): return self._rho0
    def n0(self): return self._n0
    def u0(self): return self._u0
    def molarMass0(self): return self._molarMass0


class DGFSVelocityMeshStd(_MeshBase):
    R0, NA = R0, NA

    def __init__(self, cfg):
        self.cfg = cfg
        self._nondim(cfg)
        self._S = self._L * 2.0 / (3.0 + np.sqrt(2.0))
        self._R = 2 * self._S
        self._grid()
        self._qz, self._qw = _radial_rule(cfg, self._Nrho, self._R)
        self._ssrule = cfg.lookup('spherical-design-rule', 'ssrule')
        self._M = cfg.lookupint('spherical-design-rule', 'M')
        mode = cfg.lookupordefault('spherical-design-rule', 'sphere', 'auto')
        have = {m for m, _ in available()}
        if mode == 'auto':
            mode = 'half' if 2 * self._M in have else 'full'
        if mode == 'half':
            rule = get_sphquadrule('symmetric', rule=self._ssrule,
                                   npts=2 * self._M)
            self._sz = rule.pts[0:self._M, :]
            self._sw = 2 * np.pi / self._M
            self._sphere_factor = 2.0
        elif mode == 'full':
            rule = get_sphquadrule('symmetric', rule=self._ssrule,
                                   npts=self._M)
            self._sz = rule.pts
            self._sw = 4 * np.pi / self._M
            self._sphere_factor = 1.0
        else:
            raise ValueError(f'sphere must be auto, half or full, not {mode!r}')
        self._sphere_mode = mode

    def sphere_mode(self): return self._sphere_mode


class DGFSVelocityMeshBi(_MeshBase):
    R0, NA = R0, NA

    def __init__(self, cfg):
        self.cfg = cfg
        self._nspcs = cfg.lookupint('velocity-mesh', 'nspcs')
        self._nondim(cfg)
        self._masses = [cfg.lookupfloat('velocity-mesh', 'molarMass%d' % (p + 1))
                        / self._molarMass0 for p in range(self._nspcs)]
        mr = max(self._masses)
        if mr > 4:
            raise ValueError('Mass ratio is too high!')
        self._mr = mr
        L = self._L
        self._S = min(
            L * 2.0 / (max(4. * mr / (1. + mr), 2.) + np.sqrt(1. + mr) + 1.),
            L * 2.0 / (max(4. * 1. / (1. + mr), 2.) + np.sqrt(1. + 1.0 / mr)
                       + 1.0))
        self._R = 2 * self._S
        self._grid()
        self._qz, self._qw = _radial_rule(cfg, self._Nrho, self._R)
        self._ssrule = cfg.lookup('spherical-design-rule', 'ssrule')
        self._M = cfg.lookupint('spherical-design-rule', 'M')
        self._sz = get_sphquadrule('symmetric', rule=self._ssrule,
                                   npts=self._M).pts
        self._sw = 4 * np.pi / self._M
        self._sphere_factor = 1.0

    def masses(self): return self._masses
    def nspcs(self): return self._nspcs
