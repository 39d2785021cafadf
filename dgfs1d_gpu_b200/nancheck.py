"""Blow-up check (``[dgfsnancheck] nsteps``), std/nancheck.py and
bi/nancheck.py of the reference: every ``nsteps`` steps the sum of each
solution array is read back and a NaN raises ``RuntimeError('NaNs detected
at t = ...')``.  The drivers here call it after each step when the section
is present (the reference ships the class without calling it)."""
import math


class DGFSNaNCheck:
    def __init__(self, cfg, sect='dgfsnancheck'):
        self.enabled = cfg.has_section(sect)
        self.nsteps = cfg.lookupint(sect, 'nsteps') if self.enabled else 0

    def __call__(self, tcurr, nsteps, sols):
        if not self.enabled or nsteps % self.nsteps:
            return
        for u in sols:
            if math.isnan(float(u.sum())):
                raise RuntimeError('NaNs detected at t = {0}'.format(tcurr))
