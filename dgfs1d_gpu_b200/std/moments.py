"""Bulk-moment writer of the single-species solver (``[dgfsmomwriter]``).

Moments come from the native FP64 kernel (no host copy of f); the text
output has the header and columns of dgfs1D/std/moments.py:140-220:
x, rho, U:x, U:y, T, Q:x, Q:y, P:xx, P:yy, P:xy, p, dimensional.
"""
import os

import numpy as np

FIELDS = ['rho', 'U:x', 'U:y', 'T', 'Q:x', 'Q:y', 'P:xx', 'P:yy', 'P:xy', 'p']


def dimensional(nd, vm):
    """Scale (…, 10) nondimensional moments as moments.py:61-68."""
    out = np.array(nd, dtype=np.float64, copy=True)
    rho0, u0, T0 = vm.rho0(), vm.u0(), vm.T0()
    out[..., 0:9] *= np.array([rho0, u0, u0, T0, 0.5 * rho0 * u0 ** 3,
                               0.5 * rho0 * u0 ** 3, 0.5 * rho0 * u0 ** 2,
                               0.5 * rho0 * u0 ** 2, 0.5 * rho0 * u0 ** 2])
    out[..., 9] = (vm.R0 / vm.molarMass0()) * out[..., 0] * out[..., 3]
    return out


class DGFSMomWriterStd:
    def __init__(self, cfg, vm, dg, basis, xcoeff, tcurr=None, coeff=None,
                 sect='dgfsmomwriter'):
        self.cfg, self.vm, self.dg = cfg, vm, dg
        self.enabled = cfg.has_section(sect)
        if self.enabled:
            self.basedir = cfg.lookupordefault(sect, 'basedir', '.')
            self.basename = cfg.lookup(sect, 'basename')
            if not self.basename.endswith('.txt'):
                self.basename += '.txt'
            self.dt_out = cfg.lookupfloat(sect, 'dt-out')
        im = basis.interpMat
        Nqr = im.shape[1]
        self.xsol = (im.T @ xcoeff.reshape(basis.K, -1)).reshape(Nqr, -1) \
            * vm.H0()
        self.tout_next = tcurr
        if tcurr is not None and coeff is not None:
            self(1e-10, tcurr, coeff)       # the initial state (moments.py:191)

    def compute(self, coeff):
        """(Nqr, Ne, 10) dimensional moments (host numpy)."""
        nd = self.dg.moments(coeff).cpu().numpy()
        if np.sum(nd[..., 0]) < 1e-10:      # moments.py:35-37 writes zeros
            return np.zeros_like(nd)
        return dimensional(nd, self.vm)

    def __call__(self, dt, tcurr, coeff):
        if not self.enabled:
            return None
        if self.tout_next is None:
            self.tout_next = tcurr
        if abs(self.tout_next - tcurr) > 0.5 * dt:
            return None
        sol = self.compute(coeff)
        Nqr, Ne, _ = sol.shape
        data = np.hstack((self.xsol.T.reshape(-1, 1),
                          sol.swapaxes(0, 1).reshape(Nqr * Ne, -1)))
        fname = os.path.join(self.basedir, self.basename.format(t=tcurr))
        np.savetxt(fname, data, header='t={0} \n {1}'.format(
            tcurr, ', '.join(['x0'] + FIELDS)), comments='#')
        self.tout_next = tcurr + self.dt_out
        return sol
