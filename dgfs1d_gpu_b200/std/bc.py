"""Boundary-condition plugins (``[soln-bcs-xlo|xhi] type``).

Keys and wall/inlet Maxwellians of dgfs1D/std/bc.py:9-327; the boundary
arithmetic itself runs inside the native DG right-hand side.  Each class
yields (kind, f0, ux) for ``DGOperator``.
"""
from ..plugins import subclass_where
from .initcond import DGFSMaxwellianInitConditionStd


class DGFSBCStd:
    type = None

    def __init__(self, xsol, nl, vm, cfg, cfgsect, **kwargs):
        self._vm, self.nl = vm, nl
        self.f0, self.ux = None, 0.0


class DGFSWallDiffuseBCStd(DGFSBCStd):
    type = 'dgfs-wall-diffuse'

    def __init__(self, xsol, nl, vm, cfg, cfgsect, **kwargs):
        super().__init__(xsol, nl, vm, cfg, cfgsect, **kwargs)
        ic = DGFSMaxwellianInitConditionStd(cfg, vm, cfgsect, wall=True)
        self.f0 = ic.get_init_vals()
        self.ux = float(ic.unondim()[0, 0])


class DGFSInletBCStd(DGFSBCStd):
    type = 'dgfs-inlet'

    def __init__(self, xsol, nl, vm, cfg, cfgsect, **kwargs):
        super().__init__(xsol, nl, vm, cfg, cfgsect, **kwargs)
        ic = DGFSMaxwellianInitConditionStd(cfg, vm, cfgsect)
        self.f0 = ic.get_init_vals()


class DGFSPeriodicBCStd(DGFSBCStd):
    type = 'dgfs-periodic'


def get_bc(cfg, sect, xsol, nl, vm):
    cls = subclass_where(DGFSBCStd, type=cfg.lookup(sect, 'type'))
    return cls(xsol, nl, vm, cfg, sect)
