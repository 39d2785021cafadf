"""Bulk-moment writer and residual of the binary-mixture solver.

``DGFSMomWriterBi`` (``[dgfsmomwriter]``) takes its moments from the native
FP64 mixture kernel (no host copy of f) and writes the text file of
dgfs1D/bi/moments.py:116-199: header ``t=...`` and ``x`` followed by
rho, U:x, U:y, T, Q:x, p, nden per species (suffix ``:p``), dimensional,
"%.5e".  ``DGFSResidualBi`` (``[dgfsresidual] nsteps``) records
sqrt(|u^{n+1} - u^n|^2 / |u^n|^2) per species as bi/residual.py:8-32 logs it.
"""
import math
import os

import numpy as np

FIELDS = ['rho', 'U:x', 'U:y', 'T', 'Q:x', 'p', 'nden']


def dimensional_bi(nd, vm):
    """(Nqr, Ne, nspcs, 5) nondimensional -> (Nqr, Ne, 7 nspcs) dimensional
    with pressure and number density (bi/moments.py:101-112)."""
    Nqr, Ne, ns, _ = nd.shape
    out = np.zeros((Nqr, Ne, 7 * ns))
    rho0, u0, T0, M0 = vm.rho0(), vm.u0(), vm.T0(), vm.molarMass0()
    for p, m in enumerate(vm.masses()):
        o = 7 * p
        out[:, :, o:o + 5] = nd[:, :, p, :] * np.array(
            [rho0, u0, u0, T0, 0.5 * rho0 * u0 ** 3])
        out[:, :, o + 5] = (m * vm.R0 / M0) * out[:, :, o] * out[:, :, o + 3]
        out[:, :, o + 6] = (vm.NA / m / M0) * out[:, :, o]
    return out


class DGFSMomWriterBi:
    def __init__(self, cfg, vm, dg, basis, xcoeff, tcurr=None, coeffs=None,
                 sect='dgfsmomwriter'):
        self.vm, self.dg = vm, dg
        self.enabled = cfg.has_section(sect)
        if self.enabled:
            self.basedir = cfg.lookupordefault(sect, 'basedir', '.')
            self.basename = cfg.lookup(sect, 'basename')
            if not self.basename.endswith('.txt'):
                self.basename += '.txt'
            self.dt_out = cfg.lookupfloat(sect, 'dt-out')
        fields = []
        for p in range(vm.nspcs()):
            fields += ['%s:%d' % (f, p) for f in FIELDS]
        self.fields = ', '.join(fields)
        im = basis.interpMat
        self.xsol = (np.einsum('mr,me->re', im, xcoeff).T.reshape(-1, 1)
                     * vm.H0())
        self.tout_next = tcurr
        if tcurr is not None and coeffs is not None:
            self(1e-10, tcurr, coeffs)      # the initial state, as there

    def compute(self, coeffs):
        """(Nqr, Ne, 7 nspcs) dimensional moments (host numpy)."""
        nd = self.dg.moments_bi(coeffs, self.vm.masses()).cpu().numpy()
        return dimensional_bi(nd, self.vm)

    def __call__(self, dt, tcurr, coeffs):
        if not self.enabled:
            return None
        if self.tout_next is None:
            self.tout_next = tcurr
        if abs(self.tout_next - tcurr) > 0.5 * dt:
            return None
        sol = self.compute(coeffs)
        Nqr, Ne, _ = sol.shape
        data = np.hstack((self.xsol, sol.swapaxes(0, 1).reshape(Nqr * Ne, -1)))
        fname = os.path.join(self.basedir, self.basename.format(t=tcurr))
        np.savetxt(fname, data, '%.5e',
                   header='t={0} \nx {1}'.format(tcurr, self.fields),
                   comments='#')
        self.tout_next = tcurr + self.dt_out
        return sol


class DGFSResidualBi:
    def __init__(self, cfg, dgs, sect='dgfsresidual'):
        self.dgs = dgs
        self.nsteps = int(cfg.lookupordefault(sect, 'nsteps', -1))
        self.history = []

    def __call__(self, tcurr, nsteps, prevs, currs):
        if self.nsteps <= 0 or not (nsteps % self.nsteps == 0 or nsteps == 1):
            return None
        res = []
        for dg, a, b in zip(self.dgs, currs, prevs):
            num, den = dg.residual(a, b)
            res.append(math.sqrt(num / den))
        self.history.append((tcurr, res))
        return res
