"""Expression-valued initial and boundary conditions (CPU): the expression
evaluator's rules, maxwellian-expr(-nondim) and sod-shock-tube-nondim
against direct NumPy evaluation, and the inlet/wall-expression boundary
states."""
import math

import numpy as np
import pytest

from dgfs1d_gpu_b200.config import Config, npeval
from dgfs1d_gpu_b200.configs import couette_std_ini
from dgfs1d_gpu_b200.std.initcond import get_initcond
from dgfs1d_gpu_b200.velocitymesh import DGFSVelocityMeshStd


def _ini(ics, bcs=''):
    base = couette_std_ini(Nv=16, Nrho=4).split('[soln-ics]')[0]
    return Config(base + ics + bcs)


def _xsol(Nq=3, Ne=4):
    z = np.array([-1.0, 0.0, 1.0])
    x = np.linspace(0, 1, Ne + 1)
    return np.array([0.5 * (x[j] + x[j + 1]) + 0.5 * (x[j + 1] - x[j]) * z
                     for j in range(Ne)]).T


def _mx(cv, rho, ux, uy, uz, T):
    c2 = np.sum((cv - np.array([ux, uy, uz]).reshape(3, 1)) ** 2, axis=0)
    return rho / (np.pi * T) ** 1.5 * np.exp(-c2 / T)


def test_expression_rules():
    c = Config('[a]\nx = pow(2, -1) + 3\ny = 2**3\nz = sin.__class__\n'
               'w = open(1)\n')
    assert npeval(c.lookupexpr('a', 'x'), {}) == 3.5
    with pytest.raises(ValueError):
        npeval(c.lookupexpr('a', 'y'), {})
    with pytest.raises(ValueError):
        npeval(c.lookupexpr('a', 'z'), {})
    with pytest.raises((NameError, TypeError)):
        npeval(c.lookupexpr('a', 'w'), {})
    assert np.allclose(npeval('(sin(x) + xhi)', {'x': np.array([0., 1.]), 'xhi': 2.0}),
                       [2.0, 2.0 + math.sin(1.0)])


def test_maxwellian_expr_nondim_and_dimensional():
    ics = ('[soln-ics]\ntype = maxwellian-expr-nondim\nrho = 1 + 0.1*sin(2*pi*x)\n'
           'ux = 0.05*cos(pi*x)\nuy = 0.02\nuz = 0\nT = 1 + 0.05*x\n')
    cfg = _ini(ics)
    vm = DGFSVelocityMeshStd(cfg)
    xs = _xsol()
    u = np.empty((3, 4, vm.vsize()))
    get_initcond(cfg, vm, 'soln-ics').apply_init_vals(u, 3, 4, xs)
    for q in range(3):
        for e in range(4):
            x = xs[q, e]
            ref = _mx(vm.cv(), 1 + 0.1 * math.sin(2 * math.pi * x),
                      0.05 * math.cos(math.pi * x), 0.02, 0.0, 1 + 0.05 * x)
            assert np.allclose(u[q, e], ref, rtol=1e-13, atol=0)
    # the dimensional form with the scales folded into the expressions
    dims = ('[soln-ics]\ntype = maxwellian-expr\nrho = rho0*(1 + 0.1*sin(2*pi*x))\n'
            'ux = %r*0.05*cos(pi*x)\nuy = %r*0.02\nuz = 0\nT = T0*(1 + 0.05*x)\n'
            % (float(vm.u0()), float(vm.u0())))
    cfg2 = _ini(dims)
    u2 = np.empty_like(u)
    get_initcond(cfg2, DGFSVelocityMeshStd(cfg2), 'soln-ics').apply_init_vals(u2, 3, 4, xs)
    assert np.allclose(u2, u, rtol=1e-12, atol=0)


def test_sod_nondim():
    ics = ('[soln-ics]\ntype = sod-shock-tube-nondim\nxMid = 0.5\n'
           'rho-left = 1\nT-left = 1\nux-left = 0\n'
           'rho-right = 0.125\nT-right = 0.8\nux-right = 0.1*x\n')
    cfg = _ini(ics)
    vm = DGFSVelocityMeshStd(cfg)
    xs = _xsol()
    u = np.empty((3, 4, vm.vsize()))
    get_initcond(cfg, vm, 'soln-ics').apply_init_vals(u, 3, 4, xs)
    for q in range(3):
        for e in range(4):
            x = xs[q, e]
            ref = (_mx(vm.cv(), 1.0, 0, 0, 0, 1.0) if x <= 0.5 else
                   _mx(vm.cv(), 0.125, 0.1 * x, 0, 0, 0.8))
            assert np.allclose(u[q, e], ref, rtol=1e-13, atol=0)
    bad = _ini(ics.replace('T-right = 0.8', 'T-right = 60'))
    with pytest.raises(ValueError, match='Bulk properties'):
        get_initcond(bad, DGFSVelocityMeshStd(bad), 'soln-ics').apply_init_vals(
            u, 3, 4, xs)


def test_boundary_states():
    from dgfs1d_gpu_b200.std.bc import get_bc
    bcs = ('[soln-bcs-xlo]\ntype = dgfs-inlet-nondim\nrho = 1.2\nux = 0.1\nT = 0.9\n'
           '[soln-bcs-xhi]\ntype = dgfs-wall-expr-diffuse\nT = 273\nux = 0\n'
           'uy = 50*sin(0.37*t)\nuz = 0\n')
    cfg = _ini('[soln-ics]\ntype = maxwellian\nrho = 1\nT = 273\nux = 0\nuy = 0\nuz = 0\n',
               bcs)
    vm = DGFSVelocityMeshStd(cfg)
    lo = get_bc(cfg, 'soln-bcs-xlo', 0.0, -1., vm)
    assert lo.ux == 0.1
    assert np.allclose(lo.f0, _mx(vm.cv(), 1.2, 0.1, 0, 0, 0.9), rtol=1e-14)
    hi = get_bc(cfg, 'soln-bcs-xhi', 1.0, 1., vm)
    assert hi.time_dependent
    st = hi.state(2.0)
    assert np.allclose(st, [0, 50 * math.sin(0.74) / vm.u0(), 0, 273 / vm.T0()])
    for kind in ('dgfs-cyclic', 'dgfs-vanish'):
        cfg3 = _ini('[soln-ics]\ntype = maxwellian\nrho = 1\nT = 273\nux = 0\nuy = 0\nuz = 0\n',
                    '[soln-bcs-xlo]\ntype = %s\n' % kind)
        assert get_bc(cfg3, 'soln-bcs-xlo', 0.0, -1., vm).type == kind


def test_bi_maxwellian_expr():
    from dgfs1d_gpu_b200.bi.initcond import get_initcond as get_bi
    from dgfs1d_gpu_b200.configs import couette_bi_ini
    from dgfs1d_gpu_b200.velocitymesh import DGFSVelocityMeshBi
    base = couette_bi_ini(Nv=24, Nrho=4).split('[soln-ics]')[0]
    cfg0 = Config(base + '[soln-ics]\ntype = maxwellian\nnden1 = 1\nnden2 = 1\n'
                  'T = 273\nux = 0\nuy = 0\nuz = 0\n')
    vm = DGFSVelocityMeshBi(cfg0)
    n0, u0, T0 = float(vm.n0()), float(vm.u0()), float(vm.T0())
    ics = ('[soln-ics]\ntype = maxwellian-expr\nnden1 = %r*(1 + 0.1*x)\n'
           'nden2 = %r*0.5\nux = 0\nuy = %r*0.05*sin(pi*x)\nuz = 0\n'
           'T = %r*(1 + 0.02*x)\n' % (n0, n0, u0, T0))
    cfg = Config(base + ics)
    ic = get_bi(cfg, vm, 'soln-ics')
    xs = _xsol()
    for p, m in enumerate(vm.masses()):
        u = np.empty((3, 4, vm.vsize()))
        ic.apply_init_vals(p, u, 3, 4, xs)
        for q in range(3):
            for e in range(4):
                x = xs[q, e]
                nd = (1 + 0.1 * x) if p == 0 else 0.5
                T = 1 + 0.02 * x
                c2 = np.sum((vm.cv() - np.array([0, 0.05 * math.sin(math.pi * x), 0])
                             .reshape(3, 1)) ** 2, axis=0)
                ref = nd * (m / np.pi / T) ** 1.5 * np.exp(-m * c2 / T)
                assert np.allclose(u[q, e], ref, rtol=1e-12, atol=0)
