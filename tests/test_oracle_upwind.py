"""The oracle's dgfsABUstd1D pieces against the reference's own kernels
(golden vectors: upwind operators of its basis, the explicit right-hand
side composed from std.mako / upwind.mako / boundary kernels, limitPos)."""
import os

import numpy as np

from oracle import dg as odg

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def _load():
    return np.load(os.path.join(G, 'upwind_N8.npz'))


def test_upwind_operators_match_reference_basis():
    z = _load()
    b = odg.NodalBasis('nodal-sem-gll', int(z['K']), int(z['K']))
    DpT, DmT = odg.upwind_ops(b, -1)
    assert np.allclose(DpT, z['Dp'], rtol=0, atol=1e-13)
    assert np.allclose(DmT, z['Dm'], rtol=0, atol=1e-13)
    # the package basis builds the same operators
    from dgfs1d_gpu_b200.basis import get_basis
    from dgfs1d_gpu_b200.config import Config
    from dgfs1d_gpu_b200.configs import couette_std_ini
    pb = get_basis(Config(couette_std_ini()))
    dpos, dneg = pb.upwind_ops(-1)
    assert np.allclose(dpos, z['Dm'], rtol=0, atol=1e-13)
    assert np.allclose(dneg, z['Dp'], rtol=0, atol=1e-13)


def test_upwind_rhs_matches_reference_kernels():
    z = _load()
    K, Ne, Nv = int(z['K']), int(z['Ne']), int(z['Nv'])
    b = odg.NodalBasis('nodal-sem-gll', K, K)
    cv = z['cv']
    u = z['u'].reshape(K, Ne, Nv ** 3)
    rho, ux, T = z['inlet']
    for case in ('cyclic', 'inlet_vanish'):
        if case == 'cyclic':
            bcl, bcr, swap = odg.PeriodicBC(), odg.PeriodicBC(), True
        else:
            bcl = odg.InletBC(cv, rho, T, [ux, 0, 0], -1., shift=ux)
            bcr, swap = odg.VanishBC(cv, 1.), False
        got = odg.dg_rhs_upwind(b, z['invjac'], cv[0], bcl, bcr, u, swap=swap)
        ref = z['rhs_' + case].reshape(got.shape)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), case


def test_positivity_limiter_matches_reference_kernel():
    z = _load()
    K, Ne, Nv = int(z['K']), int(z['Ne']), int(z['Nv'])
    b = odg.NodalBasis('nodal-sem-gll', K, K)
    w = z['wpos'].reshape(K, Ne, Nv ** 3)
    got = odg.limit_positivity(b, w)
    ref = z['wpos_lim'].reshape(got.shape)
    assert np.abs(got - ref).max() <= 1e-14 * np.abs(ref).max()
    assert np.abs(ref - w).max() > 0            # the limiter acted


def test_entropy_stable_rhs_matches_reference_kernels():
    z = np.load(os.path.join(G, 'entropy_N8.npz'))
    K, Ne, Nv = int(z['K']), int(z['Ne']), int(z['Nv'])
    b = odg.NodalBasis('nodal-sem-gll', K, K)
    assert np.allclose(b.derivMat, z['derivMat'], rtol=0, atol=1e-13)
    cv, cw = z['cv'], float(z['cw'])
    bcl = odg.WallDiffuseBC(cv, cw, 1.0, [0, -0.1, 0], -1.)
    bcr = odg.WallDiffuseBC(cv, cw, 1.0, [0, 0.1, 0], 1.)
    bcl.f0, bcr.f0 = z['f0L'], z['f0R']
    u = z['u'].reshape(K, Ne, Nv ** 3)
    got = odg.dg_rhs_entropy(b, z['invjac'], cv[0], bcl, bcr, u)
    ref = z['rhs'].reshape(got.shape)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    # both branches of the logarithmic mean occur
    xi = np.abs(u[0] / u[1])
    fu = ((xi - 1) / (xi + 1)) ** 2
    assert (fu < 1e-2).any() and (fu >= 1e-2).any()
