"""Single-species DGFS driver (``dgfsStd1D``) on the native kernels.

Mirrors dgfs1D/std/std.py:37-423: mesh, basis, velocity mesh, scattering
model, boundary conditions, initial condition and integrator are plugins
selected by the same INI keys; ``rhs(t, u_in, u_out)`` is the DG advection
(one native kernel pair) plus the collision operator at every (mode,
element) in one batched native call.  The solution lives on the GPU as a
(K, Ne, N^3) torch tensor; nothing is copied to the host except moments.
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
from ..velocitymesh import DGFSVelocityMeshStd
from .bc import get_bc
from .initcond import get_initcond
from .integrator import DGFSIntegratorStd
from .distributionslice import DGFSDistributionSliceStd
from .moments import DGFSMomWriterStd
from .residual import DGFSResidualStd
from .scattering import DGFSScatteringModelStd


class DGFSStd1D:
    def __init__(self, cfg, device='cuda', restart=None):
        self.cfg = cfg
        self.device = torch.device(device)
        self.dtype = torch.float64 if cfg.dtype == np.float64 else torch.float32
        self.mesh = mesh = Mesh(cfg)
        Ne = mesh.Ne
        self.basis = basis = get_basis(cfg)
        K = basis.K
        self.vm = vm = DGFSVelocityMeshStd(cfg)
        Nv = vm.vsize()
        smn = cfg.lookup('scattering-model', 'type')
        smcls = subclass_where(DGFSScatteringModelStd, scattering_model=smn)
        self.sm = smcls(cfg, vm, Ne=Ne, max_evals=K * Ne)
        ti, dt, tf = cfg.lookupfloats('time-integrator',
                                      ('tstart', 'dt', 'tend'))
        nsteps = math.ceil((tf - ti) / dt)
        self.ti, self.tf, self.nsteps = ti, tf, nsteps
        self.dt = (tf - ti) / nsteps
        x = mesh.xmesh
        self.xsol = np.array([0.5 * (x[j] + x[j + 1]) + mesh.jac[j] * basis.z
                              for j in range(Ne)]).T
        self.bcl = get_bc(cfg, 'soln-bcs-xlo', x[0], -1., vm)
        self.bcr = get_bc(cfg, 'soln-bcs-xhi', x[-1], 1., vm)
        self.dg = DGOperator(basis, mesh.invjac, vm.c0(), vm.cw(),
                             [(self.bcl.type, self.bcl.f0, self.bcl.ux),
                              (self.bcr.type, self.bcr.f0, self.bcr.ux)])
        if hasattr(self.sm, 'bind'):          # relaxation models use its tables
            self.sm.bind(self.dg)
        # collision sources: Q at mode m, element e from coefficient a
        src, dst = [], []
        for m, a in basis.mode_sources():
            for e in range(Ne):
                src.append(a * Ne + e)
                dst.append(m * Ne + e)
        self.src = torch.tensor(src, dtype=torch.int32, device=self.device)
        self.dst = torch.tensor(dst, dtype=torch.int32, device=self.device)
        # initial condition (nodal: coefficients are point values)
        usol = np.empty((basis.Nq, Ne, Nv))
        ic = get_initcond(cfg, vm, 'soln-ics')
        ic.apply_init_vals(usol, basis.Nq, Ne, self.xsol)
        self.u = torch.tensor(usol, dtype=self.dtype, device=self.device)
        if restart is not None:       # std.py:234-244
            arrs, ti = read_distribution(restart, ['coeff'], K, Ne, Nv)
            self.u.copy_(torch.from_numpy(arrs['coeff'].reshape(K, Ne, Nv)))
            self.nsteps = remaining_steps(ti, tf, self.dt)
        self.uprev = self.u.clone()
        scheme = cfg.lookup('time-integrator', 'scheme')
        icls = subclass_where(DGFSIntegratorStd, intg_kind=scheme)
        self.odes = icls(self.rhs, (K, Ne, Nv), self.dtype, device=self.device)
        self.t = ti
        self.nacptsteps = 0
        xcoeff = self.xsol  # nodal: forward transform is the identity
        self.moments = DGFSMomWriterStd(cfg, vm, self.dg, basis, xcoeff,
                                        tcurr=self.t, coeff=self.u)
        self.distribution = DGFSDistributionWriter(ti, (K, Ne, Nv), cfg)
        self.nancheck = DGFSNaNCheck(cfg)
        if cfg.has_section('dgfsdistslicewriter'):
            self.distributionslice = DGFSDistributionSliceStd(
                ti, (K, Ne, Nv), basis.interpMat, vm, cfg)
        else:
            self.distributionslice = lambda *a: None
        self.residual = DGFSResidualStd(cfg, self.dg)
        # linear slope limiter after every step (std.py:369-400)
        self.limiter = int(cfg.lookupordefault('time-integrator', 'limiter', 0))
        if self.limiter:
            self.dg.set_limiter(basis, mesh.invjac, self.xsol)

    @property
    def residuals(self):
        """[(t, residual)] recorded at step 1 and every [dgfsresidual]
        nsteps."""
        return self.residual.history

    def _advance(self):
        self.odes.integrate(self.t, self.dt, self.u)
        if self.limiter:
            self.dg.limit(self.u)

    def rhs(self, t, u_in, u_out):
        for side, bc in enumerate((self.bcl, self.bcr)):
            bc.at_time(t, self.dg, side)
        self.dg.advect(u_in, u_out)
        self.sm.fs_batch(u_in, u_out, self.src, self.dst)

    def capture_step(self):
        """Capture one time step (every RHS stage -- advection, boundary
        conditions, collision operator -- and every stage update) as one CUDA
        graph; later calls of ``step`` replay it.  A warm-up step runs first
        and is undone, so the solution is unchanged.  A boundary whose state
        depends on time (dgfs-wall-expr-diffuse) cannot be captured."""
        if self.bcl.time_dependent or self.bcr.time_dependent:
            raise ValueError('a time-dependent boundary condition cannot be '
                             'captured in a CUDA graph')
        u0 = self.u.clone()
        self._advance()
        torch.cuda.synchronize()
        self.u.copy_(u0)
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self._advance()
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        self._graph = g
        return g

    def step(self):
        if getattr(self, '_graph', None) is not None:
            self._graph.replay()
        else:
            self._advance()
        self.t += self.dt
        self.nacptsteps += 1
        self.residual(self.t, self.nacptsteps, self.u, self.uprev)
        self.moments(self.dt, self.t, self.u)
        self.distribution(self.dt, self.t, self.u)
        self.nancheck(self.t, self.nacptsteps, [self.u])
        self.distributionslice(self.dt, self.t, self.u)
        self.uprev.copy_(self.u)

    def run(self, nsteps=None):
        n = self.nsteps if nsteps is None else nsteps
        for _ in range(n):
            self.step()
        return self.u

    def bulk_moments(self):
        """(Nqr, Ne, 10) dimensional moments of the current solution."""
        return self.moments.compute(self.u)
