"""The oracle against golden vectors produced by the reference itself.

tests/golden/*.npz come from tests/golden/make_golden.py: the reference's own
setup code and its Mako CUDA kernels compiled for the CPU (cuFFT replaced by
pocketfft), on seeded inputs.
"""
import os

import numpy as np
import pytest

from oracle import collision as oc
from oracle import mesh as om

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def _load(name):
    return np.load(os.path.join(G, name))


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b))
                 / np.linalg.norm(np.ravel(b)))


@pytest.mark.parametrize('n', [2, 3, 4, 6, 8, 12, 16, 24])
def test_quadratures(n):
    g = _load('setup.npz')
    z, w = om.gauss_jacobi(n)
    assert np.allclose(z, g[f'zwgj_{n}_z'], atol=1e-15, rtol=0)
    assert np.allclose(w, g[f'zwgj_{n}_w'], atol=1e-15, rtol=0)
    z, w = om.gauss_lobatto_jacobi(n)
    assert np.allclose(z, g[f'zwglj_{n}_z'], atol=1e-15, rtol=0)
    assert np.allclose(w, g[f'zwglj_{n}_w'], atol=1e-15, rtol=0)


@pytest.mark.parametrize('cfg', [(16, 8, 6, 5.0), (32, 16, 16, 6.0),
                                 (24, 12, 6, 5.0)])
def test_velocity_mesh_and_prefactor(cfg):
    Nv, Nrho, M, dev = cfg
    g = _load('setup.npz')
    key = f'std_N{Nv}_M{M}_R{Nrho}'
    vm = om.VelocityMeshStd(Nv=Nv, M=M, Nrho=Nrho, dev=dev, rho0=0.00023)
    assert vm.L == g[key + '_L']
    assert np.allclose(vm.qz, g[key + '_qz'], rtol=1e-15, atol=0)
    assert np.allclose(vm.qw, g[key + '_qw'], rtol=1e-14, atol=0)
    assert np.array_equal(vm.sz, g[key + '_sz'])
    assert vm.sw == g[key + '_sw'] and vm.cw == g[key + '_cw']
    assert np.array_equal(vm.cv[2, :Nv], g[key + '_c0'])
    _, prefac = om.vhs_prefactor(vm, 0.81, 4.17e-10, 273.)
    assert abs(prefac / g[key + '_prefac'] - 1) < 1e-14


def _vhs_golden_tables():
    g = _load('vhs_N8.npz')
    tab = oc.VHSTables(int(g['Nv']), float(g['L']), g['qz'], g['qw'], g['sz'],
                       float(g['sw']), float(g['gamma']), sphere_factor=2.0)
    return g, tab


def test_vhs_tables_match_reference_kernels():
    g, tab = _vhs_golden_tables()
    assert _rel(tab.aa, g['aa']) < 1e-15
    assert _rel(tab.bb1, g['bb1']) < 1e-14
    assert _rel(tab.bb2, g['bb2']) < 1e-14


def test_vhs_gll_fs_matches_reference_kernels():
    g, tab = _vhs_golden_tables()
    n = int(g['Nv']) ** 3
    f = g['f'].reshape(-1, n)
    Q = g['Q_vhs_gll'].reshape(-1, n)
    for s in range(f.shape[0]):
        q = oc.vhs_gll_fs(tab, float(g['prefac']), f[s])
        assert _rel(q, Q[s]) < 1e-12, s


def test_vhs_bilinear_fs_matches_reference_kernels():
    g, tab = _vhs_golden_tables()
    n = int(g['Nv']) ** 3
    f, gg = g['f'].reshape(-1, n), g['g'].reshape(-1, n)
    Q = g['Q_vhs'].reshape(-1, n)
    for s in range(f.shape[0]):
        q = oc.vhs_fs(tab, float(g['prefac']), f[s], gg[s])
        assert _rel(q, Q[s]) < 1e-12, s


@pytest.mark.parametrize('pq', ['00', '01', '10', '11'])
def test_vss_fs_matches_reference_kernels(pq):
    g = _load('vss_N8.npz')
    p, q = int(pq[0]), int(pq[1])
    m = g['masses']
    tab = oc.VSSTables(int(g['Nv']), float(g['L']), g['qz'], g['qw'], g['sz'],
                       float(g['sw']), g['szpre'], float(g['gamma' + pq]),
                       float(g['eta' + pq]), m[q] / (m[p] + m[q]))
    assert _rel(tab.aa, g['aa']) < 1e-15
    assert _rel(tab.b, g['b' + pq]) < 1e-13
    assert _rel(tab.c, g['c' + pq]) < 1e-13
    n = int(g['Nv']) ** 3
    fp, fq = g['f%d' % p].reshape(-1, n), g['f%d' % q].reshape(-1, n)
    Q = g['Q' + pq].reshape(-1, n)
    for s in range(fp.shape[0]):
        out = oc.vss_fs(tab, float(g['prefac' + pq]), m[p], m[q], fp[s], fq[s])
        assert _rel(out, Q[s]) < 1e-12, (pq, s)


def test_vss_mesh_and_prefactors():
    g = _load('vss_N8.npz')
    vm = om.VelocityMeshBi(Nv=8, M=6, masses=list(g['masses']), Nrho=4,
                           dev=5.0, rho0=0.00011140244750324529)
    assert vm.L == g['L'] and vm.cw == g['cw']
    assert np.allclose(vm.qz, g['qz'], rtol=1e-15, atol=0)
    assert np.array_equal(vm.sz, g['sz'])
    assert np.array_equal(om.sphere_design(12), g['szpre'])
    params = {'00': (1.4, 0.81, 4.11e-10), '01': (1.36, 0.805, 4.405e-10),
              '10': (1.36, 0.805, 4.405e-10), '11': (1.32, 0.80, 4.7e-10)}
    for pq, (alpha, omega, dRef) in params.items():
        _, pf = om.vss_prefactor(vm, int(pq[0]), int(pq[1]), alpha, omega,
                                 dRef, 273.)
        assert abs(pf / g['prefac' + pq] - 1) < 1e-14
