"""Penalty models (``[penalized-scattering-model] type``) of the IMEX path.

``bgk-direct-gll`` and ``boltz-bgk-direct-gll`` keep the prefactors of
dgfs1D/astd/scattering.py:44-75 and 424-448 and the interface the
integrators call (moment, constructMaxwellian, collide, implicit update);
the arithmetic runs in the native FP64 kernels.
"""
import ctypes
from math import gamma

import numpy as np
import torch

from .. import _native as nat
from ..collision import _DT, _stream_ptr


class DGFSScatteringModelAstd:
    scattering_model = None
    nalph = 5

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

    def moment(self, t, f, U):
        npts = f.numel() // self.vm.vsize()
        nat.check(nat.lib().dgfs_penalty_moments(
            self._dg._h, ctypes.c_void_p(f.data_ptr()), _DT[f.dtype], npts,
            ctypes.c_void_p(U.data_ptr()), _stream_ptr(None)))

    def collide(self, t, U, f, P, M=None):
        npts = f.numel() // self.vm.vsize()
        nat.check(nat.lib().dgfs_penalty_collide(
            self._dg._h, ctypes.c_void_p(U.data_ptr()),
            ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(P.data_ptr()),
            ctypes.c_void_p(M.data_ptr() if M is not None else 0),
            _DT[f.dtype], npts, self._prefactor, self._omega, _stream_ptr(None)))

    def implicit(self, U, rhs, f, adiv, cdt, P=None, M=None):
        """f = (rhs + cdt nu M(U)) / (adiv + cdt nu); P = nu (M - f)."""
        npts = f.numel() // self.vm.vsize()
        nat.check(nat.lib().dgfs_penalty_implicit(
            self._dg._h, ctypes.c_void_p(U.data_ptr()),
            ctypes.c_void_p(rhs.data_ptr()), ctypes.c_void_p(f.data_ptr()),
            ctypes.c_void_p(P.data_ptr() if P is not None else 0),
            ctypes.c_void_p(M.data_ptr() if M is not None else 0),
            _DT[f.dtype], npts, float(adiv), float(cdt), self._prefactor,
            self._omega, _stream_ptr(None)))


class DGFSBGKDirectGLLScatteringModelAstd(DGFSScatteringModelAstd):
    scattering_model = 'bgk-direct-gll'

    def load_parameters(self):
        cfg, vm = self.cfg, self.vm
        omega = cfg.lookupfloat('penalized-scattering-model', 'omega')
        muRef = cfg.lookupfloat('penalized-scattering-model', 'muRef')
        Tref = cfg.lookupfloat('penalized-scattering-model', 'Tref')
        t0 = vm.H0() / vm.u0()
        visc = muRef * ((vm.T0() / Tref) ** omega)
        p0 = vm.n0() * vm.R0 / vm.NA * vm.T0()
        self._prefactor = float(t0 * p0 / visc)
        self._omega = float(omega)


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
