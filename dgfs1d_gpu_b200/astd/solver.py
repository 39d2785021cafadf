"""Penalised IMEX DGFS driver (``dgfsABstd1D``) on the native kernels.

Mirrors dgfs1D/astd/abstd.py:38-499: the Boltzmann model (``[scattering-
model]``, explicit), the penalty model (``[penalized-scattering-model]``,
implicit, FP64) and the IMEX integrator built as
``odescls(explicit, psm, shape, dtype, t=, dt=, f0=, explicitQ=)``.  The
state is kept in FP64; the Boltzmann operator may run in its FP32 mode.
"""
import math

import numpy as np
import torch

from ..basis import get_basis
from ..dg import DGOperator
from ..distribution import (DGFSDistributionWriter, read_distribution,
                            remaining_steps)
from ..mesh import Mesh
from ..nancheck import DGFSNaNCheck
from ..plugins import subclass_where
from ..std.bc import get_bc
from ..std.initcond import get_initcond
from ..std.moments import DGFSMomWriterStd
from ..std.residual import DGFSResidualStd
from ..std.scattering import DGFSScatteringModelStd
from ..velocitymesh import DGFSVelocityMeshStd
from .integrator import DGFSIntegratorAstd
from .scattering import DGFSScatteringModelAstd


class DGFSABstd1D:
    def __init__(self, cfg, device='cuda', boltzmann=None, restart=None):
        self.cfg = cfg
        self.device = torch.device(device)
        self.dtype = torch.float64
        self.mesh = mesh = Mesh(cfg)
        Ne = mesh.Ne
        self.basis = basis = get_basis(cfg)
        K = basis.K
        self.vm = vm = DGFSVelocityMeshStd(cfg)
        Nv = vm.vsize()
        self._make_models(cfg, vm, Ne, K)
        ti, dt, tf = cfg.lookupfloats('time-integrator', ('tstart', 'dt', 'tend'))
        self.nsteps = int(math.ceil((tf - ti) / dt))
        self.dt = (tf - ti) / self.nsteps
        x = mesh.xmesh
        self.xsol = np.array([0.5 * (x[j] + x[j + 1]) + mesh.jac[j] * basis.z
                              for j in range(Ne)]).T
        self.bcl = bcl = get_bc(cfg, 'soln-bcs-xlo', x[0], -1., vm)
        self.bcr = bcr = get_bc(cfg, 'soln-bcs-xhi', x[-1], 1., vm)
        self.dg = DGOperator(basis, mesh.invjac, vm.c0(), vm.cw(),
                             [(bcl.type, bcl.f0, bcl.ux),
                              (bcr.type, bcr.f0, bcr.ux)])
        self.psm.bind(self.dg)
        self._configure_dg(cfg)
        src, dst = [], []
        for m, a in basis.mode_sources():
            for e in range(Ne):
                src.append(a * Ne + e)
                dst.append(m * Ne + e)
        self.src = torch.tensor(src, dtype=torch.int32, device=self.device)
        self.dst = torch.tensor(dst, dtype=torch.int32, device=self.device)
        usol = np.empty((basis.Nq, Ne, Nv))
        get_initcond(cfg, vm, 'soln-ics').apply_init_vals(usol, basis.Nq, Ne,
                                                          self.xsol)
        self.u = torch.tensor(usol, dtype=self.dtype, device=self.device)
        if restart is not None:       # abstd.py:243-253
            arrs, ti = read_distribution(restart, ['coeff'], K, Ne, Nv)
            self.u.copy_(torch.from_numpy(arrs['coeff'].reshape(K, Ne, Nv)))
            self.nsteps = remaining_steps(ti, tf, self.dt)
        self.t = ti
        self.nacptsteps = 0
        # the Boltzmann operator may be replaced (e.g. by a surrogate)
        self.boltzmann = boltzmann
        icls = subclass_where(DGFSIntegratorAstd,
                              intg_kind=cfg.lookup('time-integrator', 'scheme'))
        self.odes = icls(self.explicit, self.psm, (K, Ne, Nv), self.dtype,
                         t=ti, dt=self.dt, f0=self.u,
                         explicitQ=self.explicitQ if self.sm is not None else None,
                         device=self.device)
        self.moments = DGFSMomWriterStd(cfg, vm, self.dg, basis, self.xsol,
                                        tcurr=self.t, coeff=self.u)
        self.distribution = DGFSDistributionWriter(ti, (K, Ne, Nv), cfg)
        self.nancheck = DGFSNaNCheck(cfg)
        self.residual = DGFSResidualStd(cfg, self.dg)
        self.uprev = self.u.clone()
        # linear slope limiter after every step (abstd.py:459, 476)
        self.limiter = int(cfg.lookupordefault('time-integrator', 'limiter', 0))
        if self.limiter:
            self.dg.set_limiter(basis, mesh.invjac, self.xsol)

    def explicit(self, t, u_in, u_out):
        for side, bc in enumerate((self.bcl, self.bcr)):
            bc.at_time(t, self.dg, side)
        self.dg.advect(u_in, u_out)

    def explicitQ(self, t, u_in, u_out):
        """Accumulate Q(u_in) into u_out (abstd.py:383-395)."""
        if self.boltzmann is not None:
            self.boltzmann(t, u_in, u_out)
        else:
            self.sm.fs_batch(u_in, u_out, self.src, self.dst)

    positivity = False      # positivity limiter after the slope limiter

    def _make_models(self, cfg, vm, Ne, K):
        """The Boltzmann model of ``[scattering-model]`` (explicit) and the
        penalty model of ``[penalized-scattering-model]`` (abstd.py:80-91)."""
        smcls = subclass_where(DGFSScatteringModelStd, scattering_model=cfg.lookup(
            'scattering-model', 'type'))
        self.sm = smcls(cfg, vm, Ne=Ne, max_evals=K * Ne)
        pcls = subclass_where(DGFSScatteringModelAstd, scattering_model=cfg.lookup(
            'penalized-scattering-model', 'type'))
        self.psm = pcls(cfg, vm, Ne=Ne, eps=self.sm.prefac)

    def _configure_dg(self, cfg):
        """Hook for variants of the spatial discretisation."""

    def step(self):
        self.odes.integrate(self.t, self.dt, self.nacptsteps, self.u)
        if self.limiter:
            self.dg.limit(self.u)
            if self.positivity:
                self.dg.limit_positivity(self.u)
        self.t += self.dt
        self.nacptsteps += 1
        # post-processing of abstd.py:480-486
        self.residual(self.t, self.nacptsteps, self.u, self.uprev)
        self.moments(self.dt, self.t, self.u)
        self.distribution(self.dt, self.t, self.u)
        self.nancheck(self.t, self.nacptsteps, [self.u])
        self.uprev.copy_(self.u)

    def run(self, nsteps=None):
        for _ in range(self.nsteps if nsteps is None else nsteps):
            self.step()
        return self.u

    def bulk_moments(self):
        return self.moments.compute(self.u)


class DGFSABUstd1D(DGFSABstd1D):
    """Upwind summation-by-parts variant (``dgfsABUstd1D``, dgfs1D/astd/
    abstdu.py:37-530): the same penalised IMEX driver with the advection
    volume term split by the sign of c_x (basis operators Dp, Dm with
    ``[basis] sigma``, default -1, read as an integer as there), periodic
    traces when the right boundary is ``dgfs-cyclic`` (one rank), and, with
    ``[time-integrator] limiter = 1``, the positivity limiter after the slope
    limiter (abstdu.py:509-510)."""
    positivity = True

    def _configure_dg(self, cfg):
        sigma = cfg.lookupordefault('basis', 'sigma', -1)
        dpos, dneg = self.basis.upwind_ops(sigma)
        self.dg.set_upwind(dpos, dneg, swap=self.bcr.type == 'dgfs-cyclic')


class DGFSABE2std1D(DGFSABstd1D):
    """Entropy-stable variant (``dgfsABE2std1D``, dgfs1D/astd/abstde2.py): the
    advection volume term is the two-point form -2 c_x sum_l Dr[k][l]
    aveL(u_k, u_l) with the logarithmic mean (eDeriv of
    astd/kernels/limiters.mako:162-195); with ``[time-integrator] limiter =
    1`` the positivity limiter follows the slope limiter (abstde2.py:492-493)."""
    positivity = True

    def _configure_dg(self, cfg):
        self.dg.set_entropy_stable(self.basis.derivMat)


class DGFSAstd1D(DGFSABstd1D):
    """Linear kinetic models (``dgfsAstd1D``, dgfs1D/astd/astd.py): the model
    of ``[scattering-model]`` is itself a penalty model (bgk-, esbgk-,
    shakov-direct-gll) solved by the same IMEX schemes, with no Boltzmann
    operator (astd.py:82-86, 388-390)."""

    def _make_models(self, cfg, vm, Ne, K):
        pcls = subclass_where(DGFSScatteringModelAstd, scattering_model=cfg.lookup(
            'scattering-model', 'type'))
        self.sm = None
        self.psm = pcls(cfg, vm, Ne=Ne)
