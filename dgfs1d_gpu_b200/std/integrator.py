"""Explicit time integrators (``[time-integrator] scheme``).

Keys, stage combinations and coefficients of dgfs1D/std/integrator.py:7-157:
``cls(rhs, (K, Ne, Nv), dtype)`` and ``integrate(t, dt, u)`` with
``rhs(t, u_in, u_out)``; stage updates run in the native axnpby kernel.
``lserk-45`` is accepted as an alias of ``lse-rk45``.
"""
import torch

from ..dg import axnpby


class DGFSIntegratorStd:
    intg_kind = None
    _nscratch = 0

    def __init__(self, rhs, shape, dtype, device='cuda', **kwargs):
        self._rhs = rhs
        tdt = torch.float64 if dtype in (torch.float64, 'double') or \
            str(dtype).endswith('float64') else torch.float32
        self.scratch = [torch.zeros(shape, dtype=tdt, device=device)
                        for _ in range(self._nscratch)]

    def integrate(self, t, dt, d_ucoeff):
        raise NotImplementedError


class EulerIntegratorStd(DGFSIntegratorStd):
    intg_kind = 'euler'
    _nscratch = 1

    def integrate(self, t, dt, u):
        r0, = self.scratch
        self._rhs(t, u, r0)
        axnpby(u, 1.0, dt, r0)


class SSPRK2IntegratorStd(DGFSIntegratorStd):
    intg_kind = 'ssp-rk2'
    _nscratch = 2

    def integrate(self, t, dt, u):
        r0, r1 = self.scratch
        self._rhs(t, u, r0)
        axnpby(r0, dt, 1.0, u)
        self._rhs(t + dt, r0, r1)
        axnpby(u, 0.5, 0.5, r0, 0.5 * dt, r1)


class SSPRK3IntegratorStd(DGFSIntegratorStd):
    intg_kind = 'ssp-rk3'
    _nscratch = 2

    def integrate(self, t, dt, u):
        r0, r1 = self.scratch
        self._rhs(t, u, r1)
        axnpby(r0, 0.0, 1.0, u, dt, r1)
        self._rhs(t + dt, r0, r1)
        axnpby(r0, 0.25, 0.75, u, 0.25 * dt, r1)
        self._rhs(t + 0.5 * dt, r0, r1)
        axnpby(u, 1.0 / 3.0, 2.0 / 3.0, r0, 2.0 / 3.0 * dt, r1)


class LSERK45IntegratorStd(DGFSIntegratorStd):
    intg_kind = 'lse-rk45'
    _nscratch = 2
    rk45a = [0.0, -567301805773.0 / 1357537059087.0,
             -2404267990393.0 / 2016746695238.0,
             -3550918686646.0 / 2091501179385.0,
             -1275806237668.0 / 842570457699.0]
    rk45b = [1432997174477.0 / 9575080441755.0,
             5161836677717.0 / 13612068292357.0,
             1720146321549.0 / 2090206949498.0,
             3134564353537.0 / 4481467310338.0,
             2277821191437.0 / 14882151754819.0]
    rk45c = [0.0, 1432997174477.0 / 9575080441755.0,
             2526269341429.0 / 6820363962896.0,
             2006345519317.0 / 3224310063776.0,
             2802321613138.0 / 2924317926251.0]

    def integrate(self, t, dt, u):
        r0, r1 = self.scratch
        for s in range(5):
            self._rhs(t + self.rk45c[s] * dt, u, r0)
            axnpby(r1, self.rk45a[s], dt, r0)
            axnpby(u, 1., self.rk45b[s], r1)


class LSERK45AliasIntegratorStd(LSERK45IntegratorStd):
    intg_kind = 'lserk-45'
