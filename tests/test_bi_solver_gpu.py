"""The native mixture solver against the oracle (few steps, FP64)."""
import numpy as np
import pytest
import torch

from dgfs1d_gpu_b200.config import Config
from dgfs1d_gpu_b200.configs import couette_bi_ini
from oracle import collision as oc
from oracle import dg as odg
from oracle import mesh as om

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b))
                 / np.linalg.norm(np.ravel(b)))


@pytest.mark.parametrize('scheme,compat', [('euler', 0), ('ssp-rk2', 0),
                                           ('ssp-rk3', 0), ('ssp-rk3', 1),
                                           ('lse-rk45', 0)])
def test_bi_steps_match_oracle(scheme, compat):
    from dgfs1d_gpu_b200 import build
    build.build()
    from dgfs1d_gpu_b200.bi.solver import DGFSBi1D
    s = DGFSBi1D(Config(couette_bi_ini(scheme=scheme, compat=compat, nsteps=2)))
    vm, sm = s.vm, s.sm
    us0 = [u.cpu().numpy().copy() for u in s.us]
    s.run(2)
    torch.cuda.synchronize()
    got = [u.cpu().numpy() for u in s.us]
    # oracle
    m = vm.masses()
    tabs = {}
    for p in range(2):
        for q in range(2):
            tabs[p, q] = oc.VSSTables(vm.Nv(), vm.L(), vm.qz(), vm.qw(), vm.sz(),
                                      vm.sw(), sm._szpre, sm._gamma[p, q],
                                      sm._eta[p, q], m[q] / (m[p] + m[q]))
    fs = lambda p, q, f, g: oc.vss_fs(tabs[p, q], sm._prefactor[p, q],
                                      m[p], m[q], f, g)
    b = odg.NodalBasis('nodal-sem-gll', s.basis.K, s.basis.K)
    cv, cw = vm.cv(), vm.cw()
    walls = []
    for p in range(2):
        wl = odg.WallDiffuseBC(cv, cw, 1.0, [0, 0, 0], -1.)
        wr = odg.WallDiffuseBC(cv, cw, 1.0, [0, 0, 0], 1.)
        wl.f0, wr.f0 = s.dgs[p]._keep['f00'], s.dgs[p]._keep['f01']
        walls.append((wl, wr))

    def rhs(p, t, us):
        return odg.dg_rhs(b, s.mesh.invjac, cv[0], walls[p][0], walls[p][1],
                          us[p], collide=odg.collide_bi(b, p, 2, fs)(us))
    us = [u.copy() for u in us0]
    t = 0.0
    for _ in range(2):
        odg.bi_integrate(scheme, rhs, t, s.dt, us, compat=bool(compat))
        t += s.dt
    for p in range(2):
        assert _rel(got[p], us[p]) < 1e-11, (scheme, p)


def test_bi_fp32_precision_mode_tracks_fp64():
    """[scattering-model] precision-mode = fp32 selects the FP32 VSS operator;
    a few steps stay within FP32 accuracy of the FP64 plugin."""
    from dgfs1d_gpu_b200 import build
    build.build()
    from dgfs1d_gpu_b200.bi.solver import DGFSBi1D
    out = {}
    for pm in ('fp64', 'fp32'):
        s = DGFSBi1D(Config(couette_bi_ini(scheme='ssp-rk2', nsteps=3,
                                           precision_mode=pm)))
        assert s.sm.operator.precision == pm
        s.run(3)
        torch.cuda.synchronize()
        out[pm] = [u.cpu().numpy() for u in s.us]
    for p in range(2):
        assert np.all(np.isfinite(out['fp32'][p]))
        assert _rel(out['fp32'][p], out['fp64'][p]) < 1e-5, p
