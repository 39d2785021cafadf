"""Penalty models (``[penalized-scattering-model] type``) of the IMEX path.

``bgk-direct-gll`` / ``boltz-bgk-direct-gll`` (BGK: Maxwellian),
``esbgk-direct-gll`` / ``boltz-esbgk-direct-gll`` (ES-BGK: anisotropic
Gaussian, 11 moments) and ``shakov-direct-gll`` / ``boltz-shakov-direct-gll``
(Shakov: Maxwellian times the heat-flux polynomial, 14 moments) keep the
prefactors of dgfs1D/astd/scattering.py:44-75, 280-400, 424-528 and the
interface the integrators call (moment, relax = the non-conserved part of
updateMoment, collide, implicit update = constructMaxwellian +
updateDistribution); the arithmetic runs in the native FP64 kernels.  As in
the reference, the model parameters come from ``[scattering-model]``; the
``boltz-esbgk`` and ``boltz-shakov`` variants use the ES-BGK / Shakov
parameters and kernels unchanged (their own parameter methods are never
called there, astd/scattering.py:489-528).
"""
import ctypes
from math import gamma

import numpy as np

from .. import _native as nat
from ..collision import _DT, _stream_ptr


class DGFSScatteringModelAstd:
    scattering_model = None
    kind = 0          # native model code: 0 BGK, 1 ES-BGK, 2 Shakov
    nalph = 5         # moments per point
    _Pr = 1.0

    def __init__(self, cfg, velocitymesh, **kwargs):
        self.cfg, self.vm = cfg, velocitymesh
        self._eps = kwargs.get('eps')
        self.load_parameters()

    def bind(self, dg):
        """Attach the DG handle whose grid tables the kernels use."""
        self._dg = dg

    @property
    def prefac(self):
        return self._prefactor

    @property
    def omega(self):
        return self._omega

    @property
    def Pr(self):
        return self._Pr

    def moment(self, t, f, U):
        """U[npts][nalph] = the model's moments of f."""
        npts = f.numel() // self.vm.vsize()
        nat.check(nat.lib().dgfs_penalty_moments_n(
            self._dg._h, ctypes.c_void_p(f.data_ptr()), _DT[f.dtype], npts,
            self.nalph, ctypes.c_void_p(U.data_ptr()), _stream_ptr(None)))

    def relax(self, U, adiv, cdt):
        """Implicit relaxation of the non-conserved moments after a BDF / LM
        moment combination (no-op for BGK)."""
        if self.kind == 0:
            return
        nat.check(nat.lib().dgfs_penalty_model_relax(
            self._dg._h, self.kind, ctypes.c_void_p(U.data_ptr()),
            U.shape[0], float(adiv), float(cdt), self._prefactor, self._omega,
            self._Pr, _stream_ptr(None)))

    def collide(self, t, U, f, P, M=None):
        npts = f.numel() // self.vm.vsize()
        nat.check(nat.lib().dgfs_penalty_model_collide(
            self._dg._h, self.kind, ctypes.c_void_p(U.data_ptr()),
            ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(P.data_ptr()),
            ctypes.c_void_p(M.data_ptr() if M is not None else 0),
            _DT[f.dtype], npts, self._prefactor, self._omega, self._Pr,
            _stream_ptr(None)))

    def implicit(self, U, rhs, f, adiv, cdt, P=None, M=None):
        """f = (rhs + cdt nu G(U)) / (adiv + cdt nu); P = nu (G - f)."""
        npts = f.numel() // self.vm.vsize()
        nat.check(nat.lib().dgfs_penalty_model_implicit(
            self._dg._h, self.kind, ctypes.c_void_p(U.data_ptr()),
            ctypes.c_void_p(rhs.data_ptr()), ctypes.c_void_p(f.data_ptr()),
            ctypes.c_void_p(P.data_ptr() if P is not None else 0),
            ctypes.c_void_p(M.data_ptr() if M is not None else 0),
            _DT[f.dtype], npts, float(adiv), float(cdt), self._prefactor,
            self._omega, self._Pr, _stream_ptr(None)))

    def _viscous(self, Pr_factor):
        """t0 Pr_factor p0 / visc from [scattering-model] omega, muRef, Tref
        (astd/scattering.py:55-66, 289-302, 339-352)."""
        cfg, vm = self.cfg, self.vm
        omega = cfg.lookupfloat('scattering-model', 'omega')
        muRef = cfg.lookupfloat('scattering-model', 'muRef')
        Tref = cfg.lookupfloat('scattering-model', 'Tref')
        t0 = vm.H0() / vm.u0()
        visc = muRef * ((vm.T0() / Tref) ** omega)
        p0 = vm.n0() * vm.R0 / vm.NA * vm.T0()
        self._prefactor = float(t0 * Pr_factor * p0 / visc)
        self._omega = float(omega)


class DGFSBGKDirectGLLScatteringModelAstd(DGFSScatteringModelAstd):
    scattering_model = 'bgk-direct-gll'

    def load_parameters(self):
        self._viscous(1.0)
        self._Pr = 1.0


class DGFSBoltzBGKDirectGLLScatteringModelAstd(DGFSScatteringModelAstd):
    scattering_model = 'boltz-bgk-direct-gll'

    def load_parameters(self):
        cfg, vm = self.cfg, self.vm
        alpha = 1.0
        omega = cfg.lookupfloat('scattering-model', 'omega')
        dRef = cfg.lookupfloat('scattering-model', 'dRef')
        Tref = cfg.lookupfloat('scattering-model', 'Tref')
        invKn = (vm.H0() * np.sqrt(2.0) * np.pi * vm.n0() * dRef * dRef
                 * pow(Tref / vm.T0(), omega - 0.5))
        self._prefactor = float(100 * invKn * alpha / (
            pow(2.0, 2 - omega + alpha) * gamma(2.5 - omega) * np.pi))
        self._omega = float(omega)
        self._Pr = 1.0


class DGFSESBGKDirectGLLScatteringModelAstd(DGFSScatteringModelAstd):
    """ES-BGK (astd/scattering.py:280-333): prefactor t0 Pr p0/visc, Pr from
    ``[scattering-model] Pr`` (default 2/3)."""
    scattering_model = 'esbgk-direct-gll'
    kind, nalph = 1, 11

    def load_parameters(self):
        self._Pr = float(self.cfg.lookupordefault('scattering-model', 'Pr',
                                                  2. / 3.))
        self._viscous(self._Pr)


class DGFSShakovDirectGLLScatteringModelAstd(DGFSScatteringModelAstd):
    """Shakov (astd/scattering.py:336-389): prefactor t0 p0/visc, Pr from
    ``[scattering-model] Pr`` (default 2/3)."""
    scattering_model = 'shakov-direct-gll'
    kind, nalph = 2, 14

    def load_parameters(self):
        self._Pr = float(self.cfg.lookupordefault('scattering-model', 'Pr',
                                                  2. / 3.))
        self._viscous(1.0)


class DGFSBoltzESBGKDirectGLLScatteringModelAstd(
        DGFSESBGKDirectGLLScatteringModelAstd):
    scattering_model = 'boltz-esbgk-direct-gll'


class DGFSBoltzShakovDirectGLLScatteringModelAstd(
        DGFSShakovDirectGLLScatteringModelAstd):
    scattering_model = 'boltz-shakov-direct-gll'
