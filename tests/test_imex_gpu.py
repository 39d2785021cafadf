"""Native penalised IMEX schemes against the oracle (FP64, few steps)."""
import numpy as np
import pytest
import torch

from dgfs1d_gpu_b200.config import Config
from dgfs1d_gpu_b200.configs import couette_astd_ini
from oracle import collision as oc
from oracle import dg as odg
from oracle import imex as oim

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b))
                 / np.linalg.norm(np.ravel(b)))


@pytest.mark.parametrize('scheme,penalty', [
    ('bdf-111', 'bgk-direct-gll'), ('bdf-222', 'bgk-direct-gll'),
    ('imex-lm-bdf1', 'boltz-bgk-direct-gll'),
    ('imex-lm-bdf2', 'boltz-bgk-direct-gll')])
def test_imex_matches_oracle(scheme, penalty):
    from dgfs1d_gpu_b200 import build
    build.build()
    from dgfs1d_gpu_b200.astd.solver import DGFSABstd1D
    ini = couette_astd_ini(scheme=scheme, penalty=penalty, Nv=8, Nrho=4,
                           nsteps=3, dt=0.002)
    s = DGFSABstd1D(Config(ini))
    f0 = s.odes.hist[0]['F'].cpu().numpy() if hasattr(s.odes, 'hist') and \
        s.odes.hist else s.u.cpu().numpy()
    f0 = np.array(f0)
    s.run(3)
    torch.cuda.synchronize()
    got = s.u.cpu().numpy()
    vm = s.vm
    b = odg.NodalBasis(s.basis.basis_kind, s.basis.K, s.basis.K)
    cv, cw = vm.cv(), vm.cw()
    bcl = odg.WallDiffuseBC(cv, cw, 1.0, [0, 0, 0], -1.)
    bcr = odg.WallDiffuseBC(cv, cw, 1.0, [0, 0, 0], 1.)
    bcl.f0, bcr.f0 = s.dg._keep['f00'], s.dg._keep['f01']
    tab = oc.VHSTables(vm.Nv(), vm.L(), vm.qz(), vm.qw(), vm.sz(), vm.sw(),
                       s.sm._gamma, sphere_factor=vm.sphere_factor())
    explicit = lambda f: odg.dg_rhs(b, s.mesh.invjac, cv[0], bcl, bcr, f)

    def boltz(f):
        out = np.zeros_like(f)
        odg.collide_fs(b, lambda x, y: oc.vhs_gll_fs(tab, s.sm.prefac, x))(f, out)
        return out
    o = oim.IMEX(scheme, explicit, boltz, cv, cw, s.psm.prefac, s.psm.omega,
                 s.dt, f0)
    f = f0.copy()
    for _ in range(3):
        f = o.step(f)
    assert _rel(got, f) < 1e-11, scheme
