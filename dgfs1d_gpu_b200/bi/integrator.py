"""Explicit integrators of the mixture solver (dgfs1D/bi/integrator.py).

``integrate(t, dt, us)`` over the list of species arrays with
``rhs(p, t, us_in, out)``.  The reference's ``ssp-rk3`` second stage
computes 0.25 dt r1 + 0.75 u + dt r0 (bi/integrator.py:128-129), which is not
SSP-RK3; the default here is the correct stage (0.25 dt r1 + 0.75 u +
0.25 r0), and ``[time-integrator] bi-ssp-rk3-compat = 1`` reproduces the
reference's.
"""
import torch

from ..dg import axnpby


class DGFSIntegratorBi:
    intg_kind = None

    def __init__(self, rhs, shape, dtype, nspcs, device='cuda', cfg=None,
                 **kwargs):
        self._rhs, self._nspcs = rhs, nspcs
        self.scratch = [torch.zeros(shape, dtype=dtype, device=device)
                        for _ in range(self._nscratch())]
        self._compat = bool(cfg.lookupordefault('time-integrator',
                                                'bi-ssp-rk3-compat', 0)) \
            if cfg is not None else False

    def _nscratch(self):
        return self._nspcs

    @staticmethod
    def copy(olds, news):
        for o, n in zip(olds, news):
            n.copy_(o)


class EulerIntegratorBi(DGFSIntegratorBi):
    intg_kind = 'euler'

    def integrate(self, t, dt, us):
        r0 = self.scratch
        for p in range(self._nspcs):
            self._rhs(p, t, us, r0[p])
            axnpby(r0[p], dt, 1.0, us[p])
        self.copy(r0, us)


class SSPRK2IntegratorBi(DGFSIntegratorBi):
    intg_kind = 'ssp-rk2'

    def _nscratch(self):
        return self._nspcs + 1

    def integrate(self, t, dt, us):
        ns = self._nspcs
        r0, r1 = self.scratch[:ns], self.scratch[ns:]
        for p in range(ns):
            self._rhs(p, t, us, r0[p])
            axnpby(r0[p], dt, 1.0, us[p])
        for p in range(ns):
            self._rhs(p, t + dt, r0, r1[0])
            axnpby(us[p], 0.5, 0.5, r0[p], 0.5 * dt, r1[0])


class SSPRK3IntegratorBi(DGFSIntegratorBi):
    intg_kind = 'ssp-rk3'

    def _nscratch(self):
        return 2 * self._nspcs

    def integrate(self, t, dt, us):
        ns = self._nspcs
        r0, r1 = self.scratch[:ns], self.scratch[ns:]
        for p in range(ns):
            self._rhs(p, t, us, r1[p])
            axnpby(r0[p], 0.0, 1.0, us[p], dt, r1[p])
        for p in range(ns):
            self._rhs(p, t + dt, r0, r1[p])
            if self._compat:
                axnpby(r1[p], 0.25 * dt, 0.75, us[p], dt, r0[p])
            else:
                axnpby(r1[p], 0.25 * dt, 0.75, us[p], 0.25, r0[p])
        for p in range(ns):
            self._rhs(p, t + 0.5 * dt, r1, r0[0])
            axnpby(us[p], 1.0 / 3.0, 2.0 / 3.0, r1[p], 2.0 / 3.0 * dt, r0[0])


class LSERK45IntegratorBi(DGFSIntegratorBi):
    intg_kind = 'lse-rk45'
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

    def _nscratch(self):
        return 2 * self._nspcs

    def integrate(self, t, dt, us):
        ns = self._nspcs
        r0, r1 = self.scratch[:ns], self.scratch[ns:]
        for s in range(5):
            for p in range(ns):
                self._rhs(p, t + self.rk45c[s] * dt, us, r0[p])
                axnpby(r1[p], self.rk45a[s], dt, r0[p])
                axnpby(r0[p], 0., 1., us[p], self.rk45b[s], r1[p])
            self.copy(r0, us)


class LSERK45AliasIntegratorBi(LSERK45IntegratorBi):
    intg_kind = 'lserk-45'
