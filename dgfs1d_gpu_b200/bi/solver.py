"""Binary-mixture DGFS driver (``dgfsBi1D``) on the native kernels.

Mirrors dgfs1D/bi/bi.py:36-389: per species p, ``rhs(p, t, us, out)`` is the
DG advection of u_p with its own wall Maxwellians plus sum_q Q_pq(u_p, u_q)
at every (mode, element), each pair in one batched native call.
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
from ..velocitymesh import DGFSVelocityMeshBi
from .bc import get_bc
from .initcond import get_initcond
from .integrator import DGFSIntegratorBi
from .moments import DGFSMomWriterBi, DGFSResidualBi
from .scattering import DGFSScatteringModelBi


class DGFSBi1D:
    def __init__(self, cfg, device='cuda', restart=None):
        self.cfg = cfg
        self.device = torch.device(device)
        self.dtype = torch.float64 if cfg.dtype == np.float64 else torch.float32
        self.mesh = mesh = Mesh(cfg)
        Ne = mesh.Ne
        self.basis = basis = get_basis(cfg)
        K = basis.K
        self.vm = vm = DGFSVelocityMeshBi(cfg)
        ns, Nv = vm.nspcs(), vm.vsize()
        self.nspcs = ns
        smcls = subclass_where(DGFSScatteringModelBi, scattering_model=cfg.lookup(
            'scattering-model', 'type'))
        self.sm = smcls(cfg, vm, Ne=Ne, max_evals=K * Ne)
        ti, dt, tf = cfg.lookupfloats('time-integrator', ('tstart', 'dt', 'tend'))
        self.nsteps = math.ceil((tf - ti) / dt)
        self.dt = (tf - ti) / self.nsteps
        x = mesh.xmesh
        self.xsol = np.array([0.5 * (x[j] + x[j + 1]) + mesh.jac[j] * basis.z
                              for j in range(Ne)]).T
        self.bcl = bcl = get_bc(cfg, 'soln-bcs-xlo', x[0], -1., vm)
        self.bcr = bcr = get_bc(cfg, 'soln-bcs-xhi', x[-1], 1., vm)
        self.dgs = [DGOperator(basis, mesh.invjac, vm.c0(), vm.cw(),
                               [(bcl.type, bcl.f0[p], bcl.ux),
                                (bcr.type, bcr.f0[p], bcr.ux)])
                    for p in range(ns)]
        src, dst = [], []
        for m, a in basis.mode_sources():
            for e in range(Ne):
                src.append(a * Ne + e)
                dst.append(m * Ne + e)
        self.src = torch.tensor(src, dtype=torch.int32, device=self.device)
        self.dst = torch.tensor(dst, dtype=torch.int32, device=self.device)
        ic = get_initcond(cfg, vm, 'soln-ics')
        self.us = []
        for p in range(ns):
            usol = np.empty((basis.Nq, Ne, Nv))
            ic.apply_init_vals(p, usol, basis.Nq, Ne, self.xsol)
            self.us.append(torch.tensor(usol, dtype=self.dtype, device=self.device))
        if restart is not None:       # bi.py:223-236
            names = ['coeff%d' % p for p in range(ns)]
            arrs, ti = read_distribution(restart, names, K, Ne, Nv)
            for u, n in zip(self.us, names):
                u.copy_(torch.from_numpy(arrs[n].reshape(K, Ne, Nv)))
            self.nsteps = remaining_steps(ti, tf, self.dt)
        icls = subclass_where(DGFSIntegratorBi,
                              intg_kind=cfg.lookup('time-integrator', 'scheme'))
        self.odes = icls(self.rhs, (K, Ne, Nv), self.dtype, ns,
                         device=self.device, cfg=cfg)
        self.t = ti
        self.nacptsteps = 0
        self.uprevs = [u.clone() for u in self.us]
        self.moments = DGFSMomWriterBi(cfg, vm, self.dgs[0], basis, self.xsol,
                                       tcurr=ti, coeffs=self.us)
        self.residual = DGFSResidualBi(cfg, self.dgs)
        self.distribution = DGFSDistributionWriter(ti, (K, Ne, Nv), cfg,
                                                   nspcs=ns)
        self.nancheck = DGFSNaNCheck(cfg)

    def rhs(self, p, t, us, out):
        for side, bc in enumerate((self.bcl, self.bcr)):
            bc.at_time(t, self.dgs[p], side, p)
        self.dgs[p].advect(us[p], out)
        self.sm.fs_batch_species(p, us, out, self.src, self.dst)

    def step(self):
        """One step and the post-processing of bi.py:360-381: residual,
        moments, then the copy of the solution for the next residual."""
        self.odes.integrate(self.t, self.dt, self.us)
        self.t += self.dt
        self.nacptsteps += 1
        self.residual(self.t, self.nacptsteps, self.uprevs, self.us)
        self.moments(self.dt, self.t, self.us)
        self.distribution(self.dt, self.t, self.us)
        self.nancheck(self.t, self.nacptsteps, self.us)
        for a, b in zip(self.uprevs, self.us):
            a.copy_(b)

    def bulk_moments(self):
        """(Nqr, Ne, 7 nspcs) dimensional mixture moments of the current
        solution (rho, U:x, U:y, T, Q:x, p, nden per species)."""
        return self.moments.compute(self.us)

    def run(self, nsteps=None):
        for _ in range(self.nsteps if nsteps is None else nsteps):
            self.step()
        return self.us
