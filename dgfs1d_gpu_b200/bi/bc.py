"""Mixture boundary conditions (dgfs1D/bi/bc.py): per-species wall/inlet
Maxwellians; the boundary arithmetic runs in the native DG kernel.
``dgfs-wall-expr-diffuse`` (bi/bc.py:122-205) evaluates its ux, uy, uz, T
expressions of t in ``at_time`` before every right-hand side; species p's
wall Maxwellian is exp(-m_p |c - u(t)|^2 / T(t))."""
from ..config import npeval
from ..plugins import subclass_where
from .initcond import DGFSMaxwellianInitConditionBi


class DGFSBCBi:
    type = None
    time_dependent = False

    def __init__(self, xsol, nl, vm, cfg, cfgsect, **kwargs):
        self.nl = nl
        self.f0 = [None] * vm.nspcs()
        self.ux = 0.0

    def at_time(self, t, dg, side, p):
        pass


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


class DGFSWallExprDiffuseBCBi(DGFSBCBi):
    type = 'dgfs-wall-expr-diffuse'
    time_dependent = True

    def __init__(self, xsol, nl, vm, cfg, cfgsect, **kwargs):
        super().__init__(xsol, nl, vm, cfg, cfgsect, **kwargs)
        self._exprs = [cfg.lookupexpr(cfgsect, k) for k in ('ux', 'uy', 'uz', 'T')]
        self._scale = [vm.u0(), vm.u0(), vm.u0(), vm.T0()]
        self._masses = list(vm.masses())
        self.state(0.0)

    def state(self, t):
        self.ux, *_ = vals = [float(npeval(e, {'t': float(t)})) / s
                              for e, s in zip(self._exprs, self._scale)]
        return vals

    def at_time(self, t, dg, side, p):
        """Hand species p's wall state at time t to its DG handle."""
        dg.set_wall_state(side, *self.state(t), mass=self._masses[p])


def get_bc(cfg, sect, xsol, nl, vm):
    cls = subclass_where(DGFSBCBi, type=cfg.lookup(sect, 'type'))
    return cls(xsol, nl, vm, cfg, sect)
