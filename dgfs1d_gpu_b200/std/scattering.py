"""Single-species scattering-model plugins (``[scattering-model] type``).

Same keys, constructor and methods as dgfs1D/std/scattering.py:18-429:
``DGFSScatteringModelStd(cfg, velocitymesh, Ne=...)`` with ``prefac``,
``omega``, ``prefacBGK/ESBGK/SK`` and ``fs(d_f, d_g, d_Q, elem, modein,
modeout)`` that *accumulates* Q into d_Q (torch CUDA tensors, slot layout
(mode*Ne + elem)*N^3 + v).  ``fs_batch`` evaluates many points in one launch.
The operator runs in the native library (FP64 parity mode or the FP32
Maxwellian-split mode, ``[scattering-model] precision-mode = fp64|fp32``,
default: fp64 for precision=double, fp32 for precision=float).
"""
import ctypes
from abc import ABCMeta, abstractmethod
from math import gamma

import numpy as np
import torch

from .. import _native as nat
from ..collision import _DT, VHSOperator, _stream_ptr
from ..dg import axnpby


class DGFSScatteringModelStd(metaclass=ABCMeta):
    scattering_model = None

    def __init__(self, cfg, velocitymesh, **kwargs):
        self.cfg = cfg
        self.vm = velocitymesh
        self.load_parameters()
        self.perform_precomputation()

    @abstractmethod
    def load_parameters(self):
        pass

    @abstractmethod
    def perform_precomputation(self):
        pass

    @abstractmethod
    def fs(self, d_arr_in, d_arr_in2, d_arr_out, elem, modein, modeout):
        pass

    @property
    def prefac(self):
        return self._prefactor

    @property
    def omega(self):
        return self._omega


class DGFSVHSGLLScatteringModelStd(DGFSScatteringModelStd):
    """VHS/HS fast-spectral Q(f,f) (std/scattering.py:51-313)."""
    scattering_model = 'vhs-gll'

    def __init__(self, cfg, velocitymesh, **kwargs):
        self._Ne = kwargs.get('Ne')
        kind = cfg.lookupordefault('basis', 'kind', 'nodal-sem-gll')
        if kind not in ('nodal-sem-gll', 'nodal-gll', 'nodal-sem-gll-2'):
            raise RuntimeError('Only tested for nodal basis')
        self._max_evals = kwargs.get('max_evals', 64)
        super().__init__(cfg, velocitymesh, **kwargs)

    @property
    def prefacBGK(self):
        return self._prefactorBGK

    @property
    def prefacESBGK(self):
        return self._prefactorESBGK

    @property
    def prefacSK(self):
        return self._prefactorSK

    def load_parameters(self):
        vm, cfg = self.vm, self.cfg
        alpha = 1.0
        omega = cfg.lookupfloat('scattering-model', 'omega')
        self._gamma = 2.0 * (1 - omega)
        dRef = cfg.lookupfloat('scattering-model', 'dRef')
        Tref = cfg.lookupfloat('scattering-model', 'Tref')
        invKn = (vm.H0() * np.sqrt(2.0) * np.pi * vm.n0() * dRef * dRef
                 * pow(Tref / vm.T0(), omega - 0.5))
        self._invKn = invKn
        self._prefactor = float(invKn * alpha / (
            pow(2.0, 2 - omega + alpha) * gamma(2.5 - omega) * np.pi))
        self._omega = omega
        Pr = cfg.lookupordefault('scattering-model', 'Pr', 2. / 3.)
        muRef = cfg.lookupordefault('scattering-model', 'muRef', 2.117e-5)
        t0 = vm.H0() / vm.u0()
        visc = muRef * ((vm.T0() / Tref) ** omega)
        p0 = vm.n0() * vm.R0 / vm.NA * vm.T0()
        self._prefactorBGK = t0 * 1.0 * p0 / visc
        self._prefactorESBGK = t0 * Pr * p0 / visc
        self._prefactorSK = self._prefactorBGK
        default = 'fp64' if cfg.dtype == np.float64 else 'fp32'
        self._precision = cfg.lookupordefault('scattering-model',
                                              'precision-mode', default)

    def perform_precomputation(self):
        vm = self.vm
        eps = 1e-15 if self.cfg.dtype == np.float64 else 1e-6
        self._op = VHSOperator(
            N=vm.Nv(), L=vm.L(), qz=vm.qz(), qw=vm.qw(), sz=vm.sz(),
            sw=vm.sw(), sphere_factor=vm.sphere_factor(), gamma=self._gamma,
            prefac=self._prefactor, cw=vm.cw(), c0=vm.c0(),
            precision=self._precision, max_evals=self._max_evals,
            sinc_eps=eps)

    @property
    def operator(self):
        return self._op

    def fs(self, d_arr_in, d_arr_in2, d_arr_out, elem, modein, modeout,
           d_nu=None):
        if d_nu is not None:
            raise NotImplementedError('collision-frequency output (d_nu)')
        Ne = self._Ne
        self._op.eval(d_arr_in, d_arr_out, src_base=modein * Ne + elem,
                      dst_base=modeout * Ne + elem, nevals=1)

    def fs_batch(self, d_f, d_Q, src, dst, stream=None):
        """Q[dst[i]] += Q(f[src[i]]) for all i in one launch sequence."""
        self._op.eval(d_f, d_Q, src=src, dst=dst, stream=stream)


class DGFSVHSScatteringModelStd(DGFSVHSGLLScatteringModelStd):
    """``vhs`` (std/scattering.py:317-429): the bilinear Q(f, g), gain from
    IFFT(cos a F) IFFT(cos a G) + IFFT(sin a F) IFFT(sin a G), loss
    f IFFT(b2 G), with f and g read at the same slot of two arrays.

    Two arrays that are the same tensor are evaluated as Q(f, f) (one pass);
    distinct arrays go through the native bilinear entry (two FP64 / three
    FP32 passes), without comparing their contents on the host.
    """
    scattering_model = 'vhs'

    @staticmethod
    def _same(a, b):
        return b is None or b is a or (
            a.data_ptr() == b.data_ptr() and a.shape == b.shape
            and a.dtype == b.dtype)

    def fs(self, d_arr_in1, d_arr_in2, d_arr_out, elem, modein, modeout,
           d_nu=None):
        if self._same(d_arr_in1, d_arr_in2):
            return super().fs(d_arr_in1, d_arr_in1, d_arr_out, elem, modein,
                              modeout, d_nu=d_nu)
        if d_nu is not None:
            raise NotImplementedError('collision-frequency output (d_nu)')
        Ne = self._Ne
        self._op.eval2(d_arr_in1, d_arr_in2, d_arr_out,
                       src_base=modein * Ne + elem,
                       dst_base=modeout * Ne + elem, nevals=1)

    def fs_batch(self, d_f, d_Q, src, dst, stream=None, d_g=None):
        """Q[dst[i]] += Q(f[src[i]], g[src[i]]) for all i (g = f if absent)."""
        if self._same(d_f, d_g):
            return super().fs_batch(d_f, d_Q, src, dst, stream=stream)
        self._op.eval2(d_f, d_g, d_Q, src=src, dst=dst, stream=stream)


class DGFSBGKDirectGLLScatteringModelStd(DGFSScatteringModelStd):
    """Explicit BGK relaxation ``bgk-direct-gll`` of dgfsStd1D
    (std/scattering.py:1186-1371, std/kernels/scattering/bgk-direct-gll.mako):
    at every point Q += prefac rho T^(1-omega) (M[rho, u, T] - f) with rho, u,
    T the moments of f there, prefac = t0 p0 / visc from ``[scattering-model]``
    omega, muRef, Tref (Pr = 1).  Runs on the native penalty kernels (moments
    and collide over all points at once); the driver binds its DG handle
    (``bind``) for the grid tables."""
    scattering_model = 'bgk-direct-gll'
    kind, nalph = 0, 5      # native penalty model: BGK, 5 moments

    def __init__(self, cfg, velocitymesh, **kwargs):
        self._Ne = kwargs.get('Ne')
        self._dg = None
        super().__init__(cfg, velocitymesh, **kwargs)

    def load_parameters(self):
        cfg, vm = self.cfg, self.vm
        omega = cfg.lookupfloat('scattering-model', 'omega')
        muRef = cfg.lookupfloat('scattering-model', 'muRef')
        Tref = cfg.lookupfloat('scattering-model', 'Tref')
        t0 = vm.H0() / vm.u0()
        visc = muRef * ((vm.T0() / Tref) ** omega)
        p0 = vm.n0() * vm.R0 / vm.NA * vm.T0()
        self._prefactor = float(t0 * 1.0 * p0 / visc)
        self._omega = float(omega)
        self._Pr = self._load_Pr()

    def _load_Pr(self):
        return 1.0

    def perform_precomputation(self):
        pass

    def bind(self, dg):
        self._dg = dg

    def _relax(self, f, Q, stream=None):
        """Q += nu (M - f) for the points (rows of N^3) of f."""
        if self._dg is None:
            raise RuntimeError('bgk-direct-gll: bind(dg) first')
        Nv = self.vm.vsize()
        npts = f.numel() // Nv
        U = torch.zeros((npts, self.nalph), dtype=torch.float64, device=f.device)
        P = torch.empty_like(f)
        sp = _stream_ptr(stream)
        nat.check(nat.lib().dgfs_penalty_moments_n(
            self._dg._h, ctypes.c_void_p(f.data_ptr()), _DT[f.dtype], npts,
            self.nalph, ctypes.c_void_p(U.data_ptr()), sp))
        nat.check(nat.lib().dgfs_penalty_model_collide(
            self._dg._h, self.kind, ctypes.c_void_p(U.data_ptr()),
            ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(P.data_ptr()),
            ctypes.c_void_p(0), _DT[f.dtype], npts, self._prefactor,
            self._omega, self._Pr, sp))
        axnpby(Q, 1.0, 1.0, P, stream=stream)

    def fs_batch(self, d_f, d_Q, src, dst, stream=None):
        """Q[dst[i]] += relaxation of f[src[i]]; the nodal bases pair every
        point with itself (src == dst).  The slot lists are inspected on the
        host once per pair of lists (the first call, before any graph
        capture)."""
        Nv = self.vm.vsize()
        f = d_f.reshape(-1, Nv)
        Q = d_Q.reshape(-1, Nv)
        key = (src.data_ptr(), dst.data_ptr(), src.numel(), f.shape[0])
        cache = self.__dict__.setdefault('_slots', {})
        if key not in cache:
            s_h, d_h = src.cpu(), dst.cpu()
            if not torch.equal(s_h, d_h):
                raise NotImplementedError('bgk-direct-gll needs src == dst slots')
            cache[key] = torch.equal(s_h.long(), torch.arange(f.shape[0]))
        if cache[key]:
            self._relax(f, Q, stream)
        else:
            idx = src.long()
            fq = f.index_select(0, idx).contiguous()
            Qq = torch.zeros_like(fq)
            self._relax(fq, Qq, stream)
            Q.index_add_(0, idx, Qq)

    def fs(self, d_arr_in, d_arr_in2, d_arr_out, elem, modein, modeout):
        Nv, Ne = self.vm.vsize(), self._Ne
        f = d_arr_in.reshape(-1, Nv)[modein * Ne + elem].reshape(1, Nv).contiguous()
        P = torch.zeros_like(f)
        self._relax(f, P)
        d_arr_out.reshape(-1, Nv)[modeout * Ne + elem] += P[0]


class DGFSShakovDirectGLLScatteringModelStd(DGFSBGKDirectGLLScatteringModelStd):
    """Explicit Shakov relaxation ``shakov-direct-gll`` of dgfsStd1D
    (std/scattering.py:1638-1846, std/kernels/scattering/shakov-direct-gll.mako):
    Q += prefac rho T^(1-omega) (M (1 + 4 (1 - Pr)/5 (q.c')/(rho T^2)
    (|c'|^2/T - 5/2)) - f), c' = c - u, q = sum f |c'|^2 c' cw, prefac =
    t0 p0 / visc and Pr from ``[scattering-model]`` (default 2/3) -- the
    Shakov collide of the penalty kernels, whose heat flux is formed from the
    raw moments."""
    scattering_model = 'shakov-direct-gll'
    kind, nalph = 2, 14

    def _load_Pr(self):
        return float(self.cfg.lookupordefault('scattering-model', 'Pr', 2. / 3.))


class DGFSESBGKDirectGLLScatteringModelStd(DGFSBGKDirectGLLScatteringModelStd):
    """Explicit ES-BGK relaxation ``esbgk-direct-gll`` of dgfsStd1D
    (std/scattering.py:1372-1637, std/kernels/scattering/esbgk-direct-gll.mako):
    Q += prefac rho / T^(omega-1) (f_ES - f) with the Gaussian f_ES whose
    covariance is the discrete second moment of (1-1/Pr) f + (1/Pr) f_M over
    rho (f_M the grid Maxwellian), prefac = t0 Pr p0 / visc and Pr from
    ``[scattering-model]`` (default 2/3).  One native kernel
    (``dgfs_std_esbgk_relax``), one block per point."""
    scattering_model = 'esbgk-direct-gll'
    kind, nalph = 1, 11

    def _load_Pr(self):
        Pr = float(self.cfg.lookupordefault('scattering-model', 'Pr', 2. / 3.))
        self._prefactor *= Pr            # t0 Pr p0 / visc
        return Pr

    def _relax(self, f, Q, stream=None):
        if self._dg is None:
            raise RuntimeError('esbgk-direct-gll: bind(dg) first')
        if f.dtype != Q.dtype or not (f.is_contiguous() and Q.is_contiguous()):
            raise ValueError('f and Q must be contiguous with the same dtype')
        npts = f.numel() // self.vm.vsize()
        nat.check(nat.lib().dgfs_std_esbgk_relax(
            self._dg._h, ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(Q.data_ptr()),
            _DT[f.dtype], npts, self._prefactor, self._omega, self._Pr,
            _stream_ptr(stream)))
