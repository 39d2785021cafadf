"""Residual of the single-species drivers (``[dgfsresidual] nsteps``).

dgfs1D/std/residual.py:9-29: at step 1 and every ``nsteps`` steps,
sqrt(|solcurr - solprev|^2 / |solprev|^2) in FP64 on the device.  The
std and abstd drivers call it as ``residual(t, n, u, u_prev)``
(std.py:407, abstd.py:481), so the norm in the denominator is that of the
new solution; the drivers here keep that call.
"""
import math


class DGFSResidualStd:
    def __init__(self, cfg, dg, sect='dgfsresidual'):
        self.dg = dg
        self.nsteps = int(cfg.lookupordefault(sect, 'nsteps', -1))
        self.history = []

    def __call__(self, tcurr, nsteps, solprev, solcurr):
        if not (self.nsteps > 0 and (nsteps % self.nsteps == 0 or nsteps == 1)):
            return None
        num, den = self.dg.residual(solcurr, solprev)   # |c - p|^2, |p|^2
        r = math.sqrt(num / den)
        self.history.append((tcurr, r))
        return r
