"""One-dimensional velocity slice of the distribution
(``[dgfsdistslicewriter]``), std/distributionslice.py:37-149.

At reconstruction point ``Nqr-out`` of element ``Ne-out`` the solution is
interpolated (interpMat) and the line of the velocity grid through the two
fixed indices given (exactly two of ``Nvx-out``, ``Nvy-out``, ``Nvz-out``)
is written every ``dt-out`` as two columns, velocity and f.  Only the K
coefficient lines of that element are read from the device.  The index
checks are against the velocity grid size N (the reference compares some of
them with the element count).
"""
import os

import numpy as np
import torch


class DGFSDistributionSliceStd:
    def __init__(self, tcurr, shape, im, vm, cfg, sect='dgfsdistslicewriter'):
        self.K, self.Ne, _ = shape
        self.vm, self.Nv = vm, vm.Nv()
        self.basedir = cfg.lookupordefault(sect, 'basedir', '.')
        self.basename = cfg.lookup(sect, 'basename')
        if not self.basename.endswith('.txt'):
            self.basename += '.txt'
        self.dt_out = cfg.lookupfloat(sect, 'dt-out')
        self.tout_next = tcurr + self.dt_out
        self.im = np.asarray(im, dtype=np.float64)
        self.Nqr = self.im.shape[1]
        self.Ne_out = int(cfg.lookup(sect, 'Ne-out'))
        self.Nqr_out = int(cfg.lookup(sect, 'Nqr-out'))
        if not 0 <= self.Ne_out < self.Ne:
            raise ValueError('Ne_out should be within [0, Ne)')
        if not 0 <= self.Nqr_out < self.Nqr:
            raise ValueError('Nqr_out should be within [0, Nqr)')
        idx = [int(cfg.lookupordefault(sect, k, -1))
               for k in ('Nvx-out', 'Nvy-out', 'Nvz-out')]
        free = [i for i, v in enumerate(idx) if v == -1]
        if len(free) == 3:
            raise ValueError('2 of the three variables (Nvx-out, Nvy-out, '
                             'Nvz-out) should be provided')
        if len(free) != 1:
            raise ValueError('Exactly 2 of the three variables (Nvx-out, '
                             'Nvy-out, Nvz-out) should be provided')
        for i, v in enumerate(idx):
            if i not in free and not 0 <= v < self.Nv:
                raise ValueError('%s should be between [0, %d)' % (
                    ('Nvx-out', 'Nvy-out', 'Nvz-out')[i], self.Nv))
        self.axis = free[0]
        N = self.Nv
        sel = [np.full(N, v) if i != self.axis else np.arange(N)
               for i, v in enumerate(idx)]
        self.vidx = (sel[0] * N + sel[1]) * N + sel[2]   # flat velocity index
        self.vslice = vm.cv()[self.axis][self.vidx]
        self._w = self.im[:, self.Nqr_out]
        self._dev_idx = None

    def line(self, coeff):
        """f at the slice (host numpy, FP64)."""
        if self._dev_idx is None or self._dev_idx.device != coeff.device:
            self._dev_idx = torch.as_tensor(self.vidx, device=coeff.device)
        rows = coeff[:, self.Ne_out, :].index_select(1, self._dev_idx)
        rows = rows.double().cpu().numpy()               # (K, N)
        return self._w @ rows

    def __call__(self, dt, tcurr, coeff):
        if abs(self.tout_next - tcurr) > 0.5 * dt:
            return None
        f = self.line(coeff)
        fname = os.path.join(self.basedir, self.basename.format(t=tcurr))
        np.savetxt(fname, np.vstack((self.vslice, f)).T, comments='#')
        self.tout_next = tcurr + self.dt_out
        return f
