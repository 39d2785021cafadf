"""The native single-species solver against the oracle and the reference."""
import os

import numpy as np
import pytest
import torch

from dgfs1d_gpu_b200.config import Config
from dgfs1d_gpu_b200.configs import couette_std_ini
from oracle import collision as oc
from oracle import dg as odg
from oracle import mesh as om

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b))
                 / np.linalg.norm(np.ravel(b)))


def _solver(ini):
    from dgfs1d_gpu_b200 import build
    build.build()
    from dgfs1d_gpu_b200.std.solver import DGFSStd1D
    return DGFSStd1D(Config(ini))


@pytest.mark.parametrize('kind', ['nodal-sem-gll', 'nodal-gll'])
def test_rhs_matches_reference_kernel_golden(kind):
    g = np.load(os.path.join(G, 'dg_%s_N8.npz' % kind.replace('-', '_')))
    ini = couette_std_ini(Ne=int(g['Ne']), K=int(g['K']), Nv=int(g['Nv']),
                          Nrho=int(g['Nrho']), M=int(g['M']), basis=kind)
    # the golden run used rho0 = 0.00023 and walls at u_y = -+0.1
    ini = ini.replace(ini.split('rho0 = ')[1].split('\n')[0], '0.00023')
    s = _solver(ini)
    assert abs(s.sm.prefac / float(g['prefac']) - 1) < 1e-14
    u = torch.tensor(g['u'].reshape(s.u.shape), device='cuda')
    out = torch.empty_like(u)
    s.rhs(0.0, u, out)
    torch.cuda.synchronize()
    assert _rel(out.cpu().numpy(), g['rhs_q']) < 1e-11


def _oracle_run(s, nsteps, scheme, limit=False):
    """Integrate the same problem with the oracle (CPU); with ``limit`` the
    slope limiter follows every step (std.py:400)."""
    vm = s.vm
    ovm = om.VelocityMeshStd(Nv=vm.Nv(), M=vm.M(), Nrho=vm.Nrho(), dev=vm.dev(),
                             rho0=vm.rho0(), full_sphere=vm.sphere_mode() == 'full')
    assert np.array_equal(ovm.sz, vm.sz())
    tab = oc.VHSTables(vm.Nv(), vm.L(), vm.qz(), vm.qw(), vm.sz(), vm.sw(),
                       s.sm._gamma, sphere_factor=vm.sphere_factor())
    b = odg.NodalBasis(s.basis.basis_kind, s.basis.K, s.basis.interpMat.shape[1])
    cv, cw = ovm.cv, ovm.cw
    bcl = odg.WallDiffuseBC(cv, cw, 1.0, [0., s.bcl.f0 is not None and
                                          -0.1 or 0, 0.], -1.)
    bcr = odg.WallDiffuseBC(cv, cw, 1.0, [0., 0.1, 0.], 1.)
    bcl.f0, bcr.f0 = s.bcl.f0, s.bcr.f0
    fs = lambda f, g: oc.vhs_gll_fs(tab, s.sm.prefac, f)
    collide = odg.collide_fs(b, fs)
    invjac = s.mesh.invjac
    u = s.u.cpu().numpy().astype(np.float64)

    def rhs(t, x):
        return odg.dg_rhs(b, invjac, cv[0], bcl, bcr, x, collide=collide)
    t = 0.0
    for _ in range(nsteps):
        odg.integrate(scheme, rhs, t, s.dt, u)
        if limit:
            u[...] = odg.limit_linear(b, invjac, s.xsol, u)
        t += s.dt
    return b, cv, cw, u


def test_couette_52_euler_steps_fp64_matches_oracle():
    """BASELINE 12-point Couette: 52 Euler steps, shear stress and heat flux
    vs the oracle to 1e-9 (FP64 mode)."""
    s = _solver(couette_std_ini())
    u0 = s.u.clone()
    b, cv, cw, uref = _oracle_run(s, 52, 'euler')
    s.u.copy_(u0)
    s.run(52)
    torch.cuda.synchronize()
    got = s.bulk_moments()   # dimensional (std/moments.py:61-68)
    vm = s.vm
    ref = odg.moments(b, uref, cv, cw, T0=vm.T0(), rho0=vm.rho0(),
                      u0=vm.u0(), molarMass0=vm.molarMass0())
    assert _rel(s.u.cpu().numpy(), uref) < 1e-11
    for i, name in ((8, 'P:xy'), (4, 'Q:x'), (5, 'Q:y'), (0, 'rho'),
                    (3, 'T')):
        assert _rel(got[:, :, i], ref[:, :, i]) < 1e-9, name


@pytest.mark.parametrize('scheme', ['ssp-rk2', 'ssp-rk3', 'lse-rk45'])
def test_integrators_match_oracle(scheme):
    s = _solver(couette_std_ini(Nv=8, Nrho=4, scheme=scheme, nsteps=3,
                                dt=0.001))
    u0 = s.u.clone()
    _, _, _, uref = _oracle_run(s, 3, scheme)
    s.u.copy_(u0)
    s.run(3)
    torch.cuda.synchronize()
    assert _rel(s.u.cpu().numpy(), uref) < 1e-11


@pytest.mark.parametrize('scheme,precision_mode', [('ssp-rk3', None),
                                                   ('lse-rk45', None),
                                                   ('ssp-rk3', 'fp32')])
def test_graph_captured_step_equals_eager_steps(scheme, precision_mode):
    """A whole time step (all RHS stages with the collision operator, the
    boundary conditions and the stage updates) captured once as a CUDA graph
    and replayed gives the eager steps' solution bit for bit."""
    ini = couette_std_ini(scheme=scheme, nsteps=6, precision_mode=precision_mode)
    a, b = _solver(ini), _solver(ini)
    b.capture_step()
    for _ in range(6):
        a.step()
        b.step()
    torch.cuda.synchronize()
    assert torch.equal(a.u, b.u)
    assert torch.isfinite(a.u).all()


def test_normal_shock_inlet_lse_rk45_graph_steps():
    """The stress configuration's set-up on a small grid: Rankine-Hugoniot
    states at Mach 1.5 joined by a tanh ramp, inlet boundaries at both ends,
    lse-rk45, FP32 operator, hard spheres; graph-captured steps equal eager
    steps bit for bit and keep the inflow/outflow densities."""
    from dgfs1d_gpu_b200.configs import normal_shock_std_ini
    ini = normal_shock_std_ini(Nv=16, Nrho=8, M=6, Ne=8, dev=8.0,
                               sphere='auto', nsteps=4)
    a, b = _solver(ini), _solver(ini)
    b.capture_step()
    for _ in range(4):
        a.step()
        b.step()
    torch.cuda.synchronize()
    assert torch.equal(a.u, b.u) and torch.isfinite(a.u).all()
    m = a.dg.moments(a.u).cpu().numpy()
    rho_l, rho_r = m[0, 0, 0], m[-1, -1, 0]
    assert abs(rho_l - 1.0) < 2e-2 and abs(rho_r - 1.714) < 3e-2, (rho_l, rho_r)


def test_std_limiter_matches_oracle():
    """dgfsStd1D with ``[time-integrator] limiter = 1``: every step followed
    by the linear slope limiter (std.py:369-400), eager and graph-captured,
    against the oracle."""
    ini = couette_std_ini(Nv=8, Nrho=4, Ne=6, scheme='ssp-rk2', nsteps=3,
                          noise=0.2)
    ini = ini.replace('[time-integrator]\n', '[time-integrator]\nlimiter = 1\n', 1)
    s = _solver(ini)
    assert s.limiter == 1
    u0 = s.u.clone()
    b, cv, cw, uref = _oracle_run(s, 3, 'ssp-rk2', limit=True)
    un = u0.cpu().numpy()
    assert np.abs(odg.limit_linear(b, s.mesh.invjac, s.xsol, un) - un).max() > 0
    s.u.copy_(u0)
    s.run(3)
    torch.cuda.synchronize()
    assert _rel(s.u.cpu().numpy(), uref) < 1e-12
    s2 = _solver(ini)
    s2.capture_step()
    s2.run(3)
    torch.cuda.synchronize()
    assert _rel(s2.u.cpu().numpy(), uref) < 1e-12


def test_std_residual_is_the_reference_norm():
    """[dgfsresidual] nsteps = 1: sqrt(|u^n - u^{n+1}|^2 / |u^{n+1}|^2), the
    normalisation the std driver's call residual(t, n, u, u_prev) gives."""
    ini = couette_std_ini(Nv=8, Nrho=4, nsteps=3) + '\n[dgfsresidual]\nnsteps = 1\n'
    s = _solver(ini)
    want = []
    for _ in range(3):
        prev = s.u.double().cpu().numpy().copy()
        s.step()
        cur = s.u.double().cpu().numpy()
        want.append(np.linalg.norm(prev - cur) / np.linalg.norm(cur))
    got = [r for _, r in s.residuals]
    assert len(got) == 3
    assert np.allclose(got, want, rtol=1e-12)


@pytest.mark.parametrize('driver', ['std', 'astd', 'bi'])
def test_restart_from_distribution_file(tmp_path, driver):
    """[dgfsdistwriter] checkpoints (datasets coeff / coeff<p> with time, K,
    Ne, Nv) and a restart from one continue the run as if uninterrupted;
    a checkpoint of another grid is refused."""
    from dgfs1d_gpu_b200 import build
    build.build()
    from dgfs1d_gpu_b200.configs import couette_astd_ini, couette_bi_ini
    if driver == 'std':
        from dgfs1d_gpu_b200.std.solver import DGFSStd1D as S
        ini = couette_std_ini(Nv=8, Nrho=4, scheme='ssp-rk3', nsteps=4)
        names = ['coeff']
    elif driver == 'astd':
        from dgfs1d_gpu_b200.astd.solver import DGFSABstd1D as S
        ini = couette_astd_ini(scheme='bdf-111', penalty='bgk-direct-gll',
                               Nv=8, Nrho=4, nsteps=4)
        names = ['coeff']
    else:
        from dgfs1d_gpu_b200.bi.solver import DGFSBi1D as S
        ini = couette_bi_ini(scheme='ssp-rk2', nsteps=4)
        names = ['coeff0', 'coeff1']
    dt = Config(ini).lookupfloat('time-integrator', 'dt')
    ini_w = ini + ('\n[dgfsdistwriter]\nbasedir = %s\nbasename = dist-{t:.6f}\n'
                   'dt-out = %.17g\n' % (tmp_path, 2 * dt))
    full = S(Config(ini))
    full.run(4)
    a = S(Config(ini_w))
    a.run(2)
    files = sorted(p.name for p in tmp_path.iterdir())
    assert len(files) == 1 and files[0].endswith('_rank=0'), files
    from dgfs1d_gpu_b200.distribution import read_distribution
    K, Ne = a.basis.K, a.mesh.Ne
    Nv = a.vm.vsize()
    arrs, t = read_distribution(str(tmp_path / files[0]), names, K, Ne, Nv)
    assert abs(t - 2 * dt) < 1e-15 and sorted(arrs) == names
    b = S(Config(ini), restart=str(tmp_path / files[0]))
    assert abs(b.t - 2 * dt) < 1e-15 and b.nsteps == 2
    b.run()
    torch.cuda.synchronize()
    ends = [full.u] if driver != 'bi' else full.us
    got = [b.u] if driver != 'bi' else b.us
    for x, y in zip(got, ends):
        assert _rel(x.cpu().numpy(), y.cpu().numpy()) < 1e-14
    with pytest.raises(ValueError, match='Inconsistent distribution'):
        S(Config(ini.replace('Ne = %d' % Ne, 'Ne = %d' % (Ne + 1), 1)),
          restart=str(tmp_path / files[0]))


def test_std_driver_writes_velocity_slice(tmp_path):
    """[dgfsdistslicewriter] in the single-species driver: the slice of the
    device solution written every dt-out equals the interpolated host copy."""
    ini = couette_std_ini(Nv=8, Nrho=4, nsteps=2)
    dt = Config(ini).lookupfloat('time-integrator', 'dt')
    ini += ('\n[dgfsdistslicewriter]\nbasedir = %s\nbasename = sl-{t:.6f}\n'
            'dt-out = %.17g\nNe-out = 1\nNqr-out = 2\nNvy-out = 3\nNvz-out = 4\n'
            % (tmp_path, dt))
    s = _solver(ini)
    s.run(2)
    torch.cuda.synchronize()
    files = sorted(tmp_path.iterdir())
    assert len(files) == 2
    N = s.vm.Nv()
    sol = np.einsum('mr,mej->rej', s.basis.interpMat,
                    s.u.cpu().numpy())[2, 1].reshape(N, N, N)[:, 3, 4]
    data = np.loadtxt(files[-1])
    assert np.allclose(data[:, 1], sol, rtol=1e-14, atol=0)
    assert np.allclose(data[:, 0], s.vm.cv()[0].reshape(N, N, N)[:, 3, 4])


def _custom_ini(ics, bcs, **kw):
    return couette_std_ini(**kw).split('[soln-ics]')[0] + ics + bcs


@pytest.mark.parametrize('case', ['inlet-vanish', 'cyclic-wallexpr'])
def test_std_expression_ics_and_boundaries_match_oracle(case):
    """maxwellian-expr-nondim / sod-shock-tube-nondim initial conditions and
    the dgfs-inlet-nondim, dgfs-vanish, dgfs-cyclic and time-dependent
    dgfs-wall-expr-diffuse boundaries in the native right-hand side, against
    the oracle over three ssp-rk2 steps (FP64)."""
    import math
    if case == 'inlet-vanish':
        ics = ('[soln-ics]\ntype = maxwellian-expr-nondim\n'
               'rho = 1 + 0.1*sin(2*pi*x)\nux = 0.05*cos(pi*x)\nuy = 0.02\n'
               'uz = 0\nT = 1 + 0.05*x\n')
        bcs = ('[soln-bcs-xlo]\ntype = dgfs-inlet-nondim\nrho = 1.1\nux = 0.2\n'
               'T = 0.95\n[soln-bcs-xhi]\ntype = dgfs-vanish\n')
    else:
        ics = ('[soln-ics]\ntype = sod-shock-tube-nondim\nxMid = 0.5\n'
               'rho-left = 1\nT-left = 1\nux-left = 0\n'
               'rho-right = 0.5\nT-right = 0.9\nux-right = 0.05*x\n')
        bcs = ('[soln-bcs-xlo]\ntype = dgfs-cyclic\n'
               '[soln-bcs-xhi]\ntype = dgfs-wall-expr-diffuse\nT = 300\nux = 0\n'
               'uy = 60*sin(2000*t)\nuz = 0\n')
    ini = _custom_ini(ics, bcs, Nv=16, Nrho=4, scheme='ssp-rk2', nsteps=3)
    s = _solver(ini)
    vm = s.vm
    u0 = s.u.cpu().numpy().copy()
    s.run(3)
    torch.cuda.synchronize()
    got = s.u.cpu().numpy()
    cv, cw = vm.cv(), vm.cw()
    if case == 'inlet-vanish':
        bcl = odg.InletBC(cv, 1.1, 0.95, [0.2, 0, 0], -1., shift=0.2)
        bcr = odg.VanishBC(cv, 1.)
    else:
        bcl = odg.PeriodicBC()
        st = lambda t: (0.0, 60 * math.sin(2000 * t) / vm.u0(), 0.0, 300 / vm.T0())
        bcr = odg.WallExprBC(cv, cw, 1., st)
    ovm = om.VelocityMeshStd(Nv=vm.Nv(), M=vm.M(), Nrho=vm.Nrho(), dev=vm.dev(),
                             rho0=vm.rho0(), full_sphere=vm.sphere_mode() == 'full')
    tab = oc.VHSTables(vm.Nv(), vm.L(), vm.qz(), vm.qw(), vm.sz(), vm.sw(),
                       s.sm._gamma, sphere_factor=vm.sphere_factor())
    b = odg.NodalBasis(s.basis.basis_kind, s.basis.K, s.basis.interpMat.shape[1])
    collide = odg.collide_fs(b, lambda f, g: oc.vhs_gll_fs(tab, s.sm.prefac, f))
    assert np.array_equal(ovm.cv, cv)

    def rhs(t, x):
        bcr.t = t
        return odg.dg_rhs(b, s.mesh.invjac, cv[0], bcl, bcr, x, collide=collide)
    u, t = u0.copy(), 0.0
    for _ in range(3):
        odg.integrate('ssp-rk2', rhs, t, s.dt, u)
        t += s.dt
    assert _rel(got, u) < 1e-11
    if case == 'cyclic-wallexpr':
        with pytest.raises(ValueError, match='time-dependent'):
            s.capture_step()


def test_command_line_run_and_restart(tmp_path, capsys):
    """``python -m dgfs1d_gpu_b200 dgfsStd1D run|restart``: a run that writes
    moments and a checkpoint, then a restart from that checkpoint that ends
    where the uninterrupted run ends."""
    from dgfs1d_gpu_b200 import build
    build.build()
    from dgfs1d_gpu_b200.__main__ import main
    ini = couette_std_ini(Nv=8, Nrho=4, nsteps=4)
    dt = Config(ini).lookupfloat('time-integrator', 'dt')
    ini += ('\n[dgfsmomwriter]\nbasedir = %s\nbasename = m-{t:.6f}\ndt-out = %.17g\n'
            '[dgfsdistwriter]\nbasedir = %s\nbasename = d-{t:.6f}\ndt-out = %.17g\n'
            % (tmp_path, 2 * dt, tmp_path, 2 * dt))
    p = tmp_path / 'run.ini'
    p.write_text(ini)
    s = main(['dgfsStd1D', 'run', str(p)])
    out = capsys.readouterr().out
    assert 'Nsteps 4' in out and 'elapsed time' in out
    names = sorted(x.name for x in tmp_path.iterdir())
    assert sum(n.startswith('m-') for n in names) == 3       # t = 0, 2dt, 4dt
    dist = sorted(n for n in names if n.startswith('d-'))
    assert len(dist) == 2
    r = main(['dgfsStd1D', 'restart', str(p), str(tmp_path / dist[0]),
              '-v', 'dgfsdistwriter::basename', 'r-{t:.6f}'])
    assert r.nsteps == 2
    assert _rel(r.u.cpu().numpy(), s.u.cpu().numpy()) < 1e-14


@pytest.mark.parametrize('model', ['bgk-direct-gll', 'shakov-direct-gll',
                                   'esbgk-direct-gll'])
def test_std_direct_relaxation_matches_oracle(model):
    """dgfsStd1D with ``[scattering-model] type = bgk-direct-gll`` /
    ``shakov-direct-gll`` (explicit relaxation at every point) over three
    ssp-rk2 steps, eager and graph-captured, against the oracle."""
    from oracle import imex as oim
    ini = couette_std_ini(Nv=8, Nrho=4, scheme='ssp-rk2', nsteps=3)
    ini = ini.replace('type = vhs-gll', 'type = %s' % model)
    s = _solver(ini)
    assert s.sm.scattering_model == model
    u0 = s.u.cpu().numpy().copy()
    s.run(3)
    torch.cuda.synchronize()
    got = s.u.cpu().numpy()
    vm = s.vm
    b = odg.NodalBasis(s.basis.basis_kind, s.basis.K, s.basis.interpMat.shape[1])
    cv, cw = vm.cv(), vm.cw()
    bcl = odg.WallDiffuseBC(cv, cw, 1.0, [0, 0, 0], -1.)
    bcr = odg.WallDiffuseBC(cv, cw, 1.0, [0, 0, 0], 1.)
    bcl.f0, bcr.f0 = s.bcl.f0, s.bcr.f0
    pre, om = s.sm.prefac, s.sm.omega

    om_model = oim.BGKModel() if s.sm.kind == 0 else oim.ShakovModel(s.sm._Pr)

    def fs(f, g):
        if s.sm.kind == 1:
            return oim.std_esbgk_relax(f, cv, cw, pre, om, s.sm._Pr)
        U = oim.moments_n(f[None], cv, cw, s.sm.nalph)
        return oim.model_collide(om_model, U, f[None], cv, pre, om).ravel()
    collide = odg.collide_fs(b, fs)
    u, t = u0.copy(), 0.0
    for _ in range(3):
        odg.integrate('ssp-rk2', lambda tt, x: odg.dg_rhs(
            b, s.mesh.invjac, cv[0], bcl, bcr, x, collide=collide), t, s.dt, u)
        t += s.dt
    assert _rel(got, u) < 1e-12
    s2 = _solver(ini)
    s2.capture_step()
    s2.run(3)
    torch.cuda.synchronize()
    assert _rel(s2.u.cpu().numpy(), got) < 1e-14


@pytest.mark.parametrize('model', ['bgk', 'shakov', 'esbgk'])
def test_std_direct_relaxation_kernel_matches_reference(model):
    """The native relaxation of one point (fs) against the golden output of
    the reference's std {bgk,shakov}-direct-gll kernels."""
    from dgfs1d_gpu_b200 import build
    build.build()
    from dgfs1d_gpu_b200.std.scattering import (
        DGFSBGKDirectGLLScatteringModelStd, DGFSESBGKDirectGLLScatteringModelStd,
        DGFSShakovDirectGLLScatteringModelStd)
    from dgfs1d_gpu_b200.basis import get_basis
    from dgfs1d_gpu_b200.dg import DGOperator
    g = np.load(os.path.join(G, 'std_relax_N8.npz'))
    N = int(g['Nv'])
    cls = {'bgk': DGFSBGKDirectGLLScatteringModelStd,
           'shakov': DGFSShakovDirectGLLScatteringModelStd,
           'esbgk': DGFSESBGKDirectGLLScatteringModelStd}[model]
    sm = object.__new__(cls)            # parameters from the golden case
    sm._Ne, sm._prefactor, sm._omega = 1, float(g['prefac']), float(g['omega'])
    sm._Pr = 1.0 if model == 'bgk' else float(g['Pr'])
    sm.vm = type('VM', (), {'vsize': lambda self: N ** 3})()
    b = get_basis(Config(couette_std_ini()))
    dg = DGOperator(b, np.ones(1), g['cv'][2, :N], float(g['cw']),
                    [('dgfs-periodic', None, 0.0), ('dgfs-periodic', None, 0.0)])
    sm.bind(dg)
    f = torch.tensor(g['f'].reshape(1, -1), device='cuda')
    Q = torch.zeros_like(f)
    sm.fs(f, f, Q, 0, 0, 0)
    torch.cuda.synchronize()
    assert _rel(Q.cpu().numpy().ravel(), g['Q_' + model]) < 1e-12
