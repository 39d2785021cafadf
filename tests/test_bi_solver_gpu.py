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


def _golden_moments():
    import os
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                'golden', 'moments_N8.npz'))


def _moment_dg(z, cv, cw):
    """A DG handle on the golden grid (K=3, Ne=4, 8^3 velocities) whose
    interpolation matrix is the reference basis' one."""
    import types
    from dgfs1d_gpu_b200.basis import get_basis
    from dgfs1d_gpu_b200.configs import couette_std_ini
    from dgfs1d_gpu_b200.dg import DGOperator
    im = z['interpMat']
    K = im.shape[0]
    Ne = z['std_f'].shape[1]
    b = get_basis(Config(couette_std_ini()))
    assert b.K == K
    nb = types.SimpleNamespace(**{k: getattr(b, k) for k in (
        'K', 'faceOp', 'derivOp', 'gLD', 'gRD', 'invMassOp')}, interpMat=im)
    N = round(cv.shape[1] ** (1 / 3))
    return DGOperator(nb, np.ones(Ne), cv[2, :N], float(cw),
                      [('dgfs-periodic', None, 0.0), ('dgfs-periodic', None, 0.0)])


def _colmax_rel(got, ref):
    scale = np.abs(ref).max(axis=(0, 1))
    scale[scale == 0] = 1.0
    return float((np.abs(got - ref).max(axis=(0, 1)) / scale).max())


def test_native_std_moments_match_reference_writer():
    """dgfs_dg_moments + the dimensional scaling against the reference's
    DGFSMomWriterStd on the golden input."""
    from dgfs1d_gpu_b200 import build
    build.build()
    from dgfs1d_gpu_b200.std.moments import dimensional
    z = _golden_moments()
    dg = _moment_dg(z, z['std_cv'], z['std_cw'])
    f = torch.tensor(z['std_f'], device='cuda')
    nd = dg.moments(f).cpu().numpy()
    vm = type('VM', (), dict(rho0=lambda s: float(z['std_rho0']),
                             u0=lambda s: float(z['std_u0']),
                             T0=lambda s: float(z['std_T0']),
                             molarMass0=lambda s: float(z['std_molarMass0']),
                             R0=8.3144598))()
    got = dimensional(nd, vm)
    assert _colmax_rel(got, z['std_mom']) < 1e-12


@pytest.mark.parametrize('tag', ['mix', 'absent'])
@pytest.mark.parametrize('dtype', [torch.float64, torch.float32])
def test_native_bi_moments_match_reference_writer(tag, dtype):
    """dgfs_dg_moments_bi + the dimensional scaling against the reference's
    DGFSMomWriterBi on the golden input: a two-species mixture, and the same
    with the second species absent (zero density: its columns stay zero and
    it is left out of the mixture velocity).  FP32 solutions are read as
    stored and summed in FP64."""
    from dgfs1d_gpu_b200 import build
    build.build()
    from dgfs1d_gpu_b200.bi.moments import dimensional_bi
    z = _golden_moments()
    dg = _moment_dg(z, z['bi_cv'], z['bi_cw'])
    fs = [z['bi_%s_f%d' % (tag, p)] for p in range(2)]
    us = [torch.tensor(f, dtype=dtype, device='cuda') for f in fs]
    nd = dg.moments_bi(us, list(z['bi_masses'])).cpu().numpy()
    vm = type('VM', (), dict(rho0=lambda s: float(z['bi_rho0']),
                             u0=lambda s: float(z['bi_u0']),
                             T0=lambda s: float(z['bi_T0']),
                             molarMass0=lambda s: float(z['bi_molarMass0']),
                             masses=lambda s: list(z['bi_masses']),
                             R0=float(z['bi_R0']), NA=float(z['bi_NA'])))()
    got = dimensional_bi(nd, vm)
    if dtype == torch.float64:
        assert _colmax_rel(got, z['bi_%s_mom' % tag]) < 1e-12
    else:
        # the reference writer on the FP32-rounded input, restated
        class B:
            interpMat = z['interpMat']
        ref = odg.moments_bi(B, [f.astype(np.float32).astype(np.float64) for f in fs],
                             z['bi_cv'], float(z['bi_cw']), list(z['bi_masses']),
                             T0=float(z['bi_T0']), rho0=float(z['bi_rho0']),
                             u0=float(z['bi_u0']), R0=float(z['bi_R0']),
                             NA=float(z['bi_NA']),
                             molarMass0=float(z['bi_molarMass0']))
        assert _colmax_rel(got, ref) < 1e-12
    if tag == 'absent':
        assert np.all(got[:, :, 7:] == 0)


def test_bi_solver_moment_file_and_residual(tmp_path):
    """The mixture driver writes the reference's moment file (initial state
    and every dt-out) and records per-species residuals; the written values
    equal the oracle's mixture moments of the solution."""
    from dgfs1d_gpu_b200 import build
    build.build()
    from dgfs1d_gpu_b200.bi.solver import DGFSBi1D
    ini = couette_bi_ini(scheme='euler', nsteps=3)
    dt = Config(ini).lookupfloat('time-integrator', 'dt')
    ini += ('\n[dgfsmomwriter]\nbasedir = %s\nbasename = mom-{t:.4e}\n'
            'dt-out = %.17g\n[dgfsresidual]\nnsteps = 1\n') % (tmp_path, float(dt))
    s = DGFSBi1D(Config(ini))
    files0 = sorted(tmp_path.iterdir())
    assert len(files0) == 1                      # the initial state
    s.run(3)
    torch.cuda.synchronize()
    files = sorted(tmp_path.iterdir())
    assert len(files) == 4
    assert len(s.residual.history) == 3
    assert all(len(r) == 2 and all(np.isfinite(r)) for _, r in s.residual.history)
    last = tmp_path / s.moments.basename.format(t=s.t)
    head = last.read_text().splitlines()[:2]
    assert head[0] == '#t=%s ' % s.t
    assert head[1] == '#x ' + ', '.join(
        '%s:%d' % (f, p) for p in range(2)
        for f in ('rho', 'U:x', 'U:y', 'T', 'Q:x', 'p', 'nden'))
    data = np.loadtxt(last)
    vm = s.vm
    ref = odg.moments_bi(s.basis, [u.cpu().numpy() for u in s.us], vm.cv(),
                         vm.cw(), vm.masses(), T0=vm.T0(), rho0=vm.rho0(),
                         u0=vm.u0(), R0=vm.R0, NA=vm.NA,
                         molarMass0=vm.molarMass0())
    Nqr, Ne, ncol = ref.shape
    ref = ref.swapaxes(0, 1).reshape(Nqr * Ne, ncol)
    assert data.shape == (Nqr * Ne, 1 + ncol)
    scale = np.abs(ref).max(axis=0)
    scale[scale == 0] = 1
    # the file keeps 6 significant digits ("%.5e")
    assert (np.abs(data[:, 1:] - ref).max(axis=0) / scale).max() < 1e-5
