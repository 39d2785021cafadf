"""The DG oracle against the reference's own std.mako / wall kernels."""
import os

import numpy as np
import pytest

from oracle import collision as oc
from oracle import dg

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b))
                 / np.linalg.norm(np.ravel(b)))


@pytest.mark.parametrize('kind', ['nodal-sem-gll', 'nodal-gll'])
def test_basis_matches_reference(kind):
    g = np.load(os.path.join(G, 'setup.npz'))
    key = 'basis_' + kind.replace('-', '_')
    b = dg.NodalBasis(kind, 3, 8)
    assert np.allclose(b.z, g[key + '_z'], atol=1e-15)
    assert np.allclose(b.gLD, g[key + '_gLD'], atol=1e-13)
    assert np.allclose(b.gRD, g[key + '_gRD'], atol=1e-13)
    assert np.allclose(b.derivMat, g[key + '_derivMat'], atol=1e-13)
    assert np.allclose(b.interpMat, g[key + '_interpMat'], atol=1e-13)
    assert np.allclose(np.stack(b.U), g[key + '_U'], atol=1e-13)
    assert np.allclose(np.stack(b.V), g[key + '_V'], atol=1e-13)
    assert np.array_equal(np.array([list(s) for s in b.sigModes]),
                          g[key + '_sigModes'])


@pytest.mark.parametrize('kind', ['nodal-sem-gll', 'nodal-gll'])
def test_rhs_matches_reference_kernels(kind):
    g = np.load(os.path.join(G, 'dg_%s_N8.npz' % kind.replace('-', '_')))
    K, Ne, N = int(g['K']), int(g['Ne']), int(g['Nv'])
    b = dg.NodalBasis(kind, K, 8)
    cv, cw = g['cv'], float(g['cw'])
    u = g['u'].reshape(K, Ne, N ** 3)
    bcl = dg.WallDiffuseBC(cv, cw, 1.0, [0., -0.1, 0.], -1.)
    bcr = dg.WallDiffuseBC(cv, cw, 1.0, [0., 0.1, 0.], 1.)
    r = dg.dg_rhs(b, g['invjac'], cv[0], bcl, bcr, u)
    assert _rel(r, g['rhs_adv']) < 1e-13
    tab = oc.VHSTables(N, float(g['L']), g['qz'], g['qw'], g['sz'],
                       float(g['sw']), float(g['gamma']), sphere_factor=2.0)
    fs = lambda f, gg: oc.vhs_gll_fs(tab, float(g['prefac']), f)
    r = dg.dg_rhs(b, g['invjac'], cv[0], bcl, bcr, u,
                  collide=dg.collide_fs(b, fs))
    assert _rel(r, g['rhs_q']) < 1e-12
