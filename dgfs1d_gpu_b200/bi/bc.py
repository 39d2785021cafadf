"""Mixture boundary conditions (dgfs1D/bi/bc.py): per-species wall/inlet
Maxwellians; the boundary arithmetic runs in the native DG kernel."""
from ..plugins import subclass_where
from .initcond import DGFSMaxwellianInitConditionBi


class DGFSBCBi:
    type = None

    def __init__(self, xsol, nl, vm, cfg, cfgsect, **kwargs):
        self.nl = nl
        self.f0 = [None] * vm.nspcs()
        self.ux = 0.0


class DGFSWallDiffuseBCBi(DGFSBCBi):
    type = 'dgfs-wall-diffuse'

    def __init__(self, xsol, nl, vm, cfg, cfgsect, **kwargs):
        super().__init__(xsol, nl, vm, cfg, cfgsect, **kwargs)
        ic = DGFSMaxwellianInitConditionBi(cfg, vm, cfgsect, wall=True)
        self.f0 = ic.get_init_vals()
        self.ux = float(ic.unondim()[0, 0])


class DGFSInletBCBi(DGFSBCBi):
    type = 'dgfs-inlet'

    def __init__(self, xsol, nl, vm, cfg, cfgsect, **kwargs):
        super().__init__(xsol, nl, vm, cfg, cfgsect, **kwargs)
        self.f0 = DGFSMaxwellianInitConditionBi(cfg, vm, cfgsect).get_init_vals()


class DGFSPeriodicBCBi(DGFSBCBi):
    type = 'dgfs-periodic'


def get_bc(cfg, sect, xsol, nl, vm):
    cls = subclass_where(DGFSBCBi, type=cfg.lookup(sect, 'type'))
    return cls(xsol, nl, vm, cfg, sect)
