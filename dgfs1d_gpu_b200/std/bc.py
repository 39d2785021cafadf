"""Boundary-condition plugins (``[soln-bcs-xlo|xhi] type``).

Keys and wall/inlet Maxwellians of dgfs1D/std/bc.py:9-327; the boundary
arithmetic itself runs inside the native DG right-hand side.  Each class
yields (kind, f0, ux) for ``DGOperator``.  ``dgfs-wall-expr-diffuse`` has
wall velocity and temperature expressions of the time ``t``; the driver calls
``at_time`` before every right-hand side, which evaluates them and hands the
state to the native kernel (``time_dependent`` is then True).
"""
import numpy as np

from ..config import npeval
from ..plugins import subclass_where
from .initcond import DGFSMaxwellianInitConditionStd


class DGFSBCStd:
    type = None
    time_dependent = False

    def __init__(self, xsol, nl, vm, cfg, cfgsect, **kwargs):
        self._vm, self.nl = vm, nl
        self.f0, self.ux = None, 0.0

    def at_time(self, t, dg, side):
        pass


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


class DGFSCyclicBCStd(DGFSBCStd):
    """One rank: the ghost state is the interior trace, as for
    ``dgfs-periodic`` (dgfs-cyclic.mako)."""
    type = 'dgfs-cyclic'


class DGFSVanishBCStd(DGFSBCStd):
    """Ghost 0 where c_x n >= 0, the interior trace elsewhere
    (dgfs-vanish.mako)."""
    type = 'dgfs-vanish'


class DGFSInletNonDimBCStd(DGFSBCStd):
    """Inlet Maxwellian from nondimensional rho, ux, T (bc.py:269-327),
    entering where (c_x - ux) n < 0; its density must be resolved by the
    grid (atol 1e-5)."""
    type = 'dgfs-inlet-nondim'

    def __init__(self, xsol, nl, vm, cfg, cfgsect, **kwargs):
        super().__init__(xsol, nl, vm, cfg, cfgsect, **kwargs)
        rho, ux, T = (cfg.lookupfloat(cfgsect, k) for k in ('rho', 'ux', 'T'))
        u = np.array([ux, 0.0, 0.0]).reshape(3, 1)
        f0 = rho / (np.pi * T) ** 1.5 * np.exp(-np.sum((vm.cv() - u) ** 2, axis=0) / T)
        if not np.allclose(rho, np.sum(f0) * vm.cw(), atol=1e-5):
            raise ValueError('Bulk properties not conserved! Check Nv, dev')
        self.f0, self.ux = f0, float(ux)


class DGFSWallExprDiffuseBCStd(DGFSBCStd):
    """Diffuse wall whose ux, uy, uz, T (dimensional) are expressions of t
    (bc.py:136-199): the unnormalised Maxwellian exp(-|c - u(t)|^2 / T(t))
    scaled by the wall density of the flux balance."""
    type = 'dgfs-wall-expr-diffuse'
    time_dependent = True
    mass = 1.0

    def __init__(self, xsol, nl, vm, cfg, cfgsect, **kwargs):
        super().__init__(xsol, nl, vm, cfg, cfgsect, **kwargs)
        self._exprs = [cfg.lookupexpr(cfgsect, k) for k in ('ux', 'uy', 'uz', 'T')]
        self._scale = [vm.u0(), vm.u0(), vm.u0(), vm.T0()]
        self.state(0.0)

    def state(self, t):
        """(ux, uy, uz, T) nondimensional at time t."""
        self.ux, *_ = vals = [float(npeval(e, {'t': float(t)})) / s
                              for e, s in zip(self._exprs, self._scale)]
        return vals

    def at_time(self, t, dg, side):
        dg.set_wall_state(side, *self.state(t), mass=self.mass)


def get_bc(cfg, sect, xsol, nl, vm):
    cls = subclass_where(DGFSBCStd, type=cfg.lookup(sect, 'type'))
    return cls(xsol, nl, vm, cfg, sect)
