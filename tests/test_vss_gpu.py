"""Parity of the CUDA VSS mixture operator with the reference and the oracle."""
import os

import numpy as np
import pytest
import torch

from oracle import collision as oc
from oracle import mesh as om

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
FP32_TOL = 1e-5   # relative L2, FP32 mode (Maxwellian split)
FP64_TOL = 1e-11


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b))
                 / np.linalg.norm(np.ravel(b)))


@pytest.fixture(scope='module')
def built():
    from dgfs1d_gpu_b200 import build
    build.build()


def _op_from(g, max_evals=8):
    from dgfs1d_gpu_b200.collision import VSSOperator
    pairs = ['00', '01', '10', '11']
    gam = np.array([float(g['gamma' + pq]) for pq in pairs]).reshape(2, 2)
    eta = np.array([float(g['eta' + pq]) for pq in pairs]).reshape(2, 2)
    pre = np.array([float(g['prefac' + pq]) for pq in pairs]).reshape(2, 2)
    return VSSOperator(int(g['Nv']), float(g['L']), g['qz'], g['qw'], g['sz'],
                       float(g['sw']), g['szpre'], g['masses'], gam, eta, pre,
                       max_evals=max_evals)


@pytest.mark.parametrize('pq', ['00', '01', '10', '11'])
def test_vss_matches_reference_kernel_golden(built, pq):
    g = np.load(os.path.join(G, 'vss_N8.npz'))
    op = _op_from(g)
    p, q = int(pq[0]), int(pq[1])
    fs = [torch.tensor(g['f0'], device='cuda'), torch.tensor(g['f1'], device='cuda')]
    Q = torch.zeros_like(fs[p])
    op.eval(p, q, fs[p], fs[q], Q)
    torch.cuda.synchronize()
    n = int(g['Nv']) ** 3
    ref = g['Q' + pq].reshape(-1, n)
    got = Q.cpu().numpy().reshape(-1, n)
    for s in range(ref.shape[0]):
        assert _rel(got[s], ref[s]) < FP64_TOL, (pq, s)


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
@pytest.mark.parametrize('N', [16, 24])
def test_vss_matches_oracle(built, N, precision):
    from dgfs1d_gpu_b200.collision import VSSOperator
    masses = [1.0, 2.0]
    vm = om.VelocityMeshBi(Nv=N, M=6, masses=masses, Nrho=6, dev=5.0)
    szpre = om.sphere_design(32)
    rng = np.random.default_rng(5)
    cv = vm.cv
    f = []
    for sp, T in ((0, 1.0), (1, 1.2)):
        m = 0.5 * np.exp(-np.sum(cv ** 2, axis=0) / T) / (np.pi * T) ** 1.5
        f.append(m * (1 + 0.02 * rng.uniform(-1, 1, m.shape)))
    alpha, omega = 1.4, 0.81
    gam = np.full((2, 2), 2 * (1 - omega))
    eta = np.full((2, 2), alpha - 1)
    pre = np.array([[0.1, 0.11], [0.12, 0.13]])
    op = VSSOperator(N, vm.L, vm.qz, vm.qw, vm.sz, vm.sw, szpre, masses, gam,
                     eta, pre, max_evals=2, precision=precision)
    fd = [torch.tensor(x[None], device='cuda') for x in f]
    tol = FP64_TOL if precision == 'fp64' else FP32_TOL
    for p, q in ((0, 1), (1, 1)):
        tab = oc.VSSTables(N, vm.L, vm.qz, vm.qw, vm.sz, vm.sw, szpre,
                           gam[p, q], eta[p, q], masses[q] / (masses[p] + masses[q]))
        ref = oc.vss_fs(tab, pre[p, q], masses[p], masses[q], f[p], f[q])
        Q = torch.zeros_like(fd[p])
        op.eval(p, q, fd[p], fd[q], Q)
        torch.cuda.synchronize()
        err = _rel(Q.cpu().numpy()[0], ref)
        assert err < tol, (N, p, q, precision, err)


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
@pytest.mark.parametrize('N', [16, 24])
def test_vss_species_sum_matches_oracle(built, N, precision):
    """dgfs_vss_eval_species: every pair of species p in one call,
    Q_p += sum_q Q_pq(f_p, f_q), slot lists and += included."""
    from dgfs1d_gpu_b200.collision import VSSOperator
    masses = [1.0, 2.0]
    vm = om.VelocityMeshBi(Nv=N, M=6, masses=masses, Nrho=6, dev=5.0)
    szpre = om.sphere_design(32)
    rng = np.random.default_rng(7)
    cv = vm.cv
    f = []
    for sp, T in ((0, 1.0), (1, 1.2)):
        m = 0.5 * np.exp(-np.sum(cv ** 2, axis=0) / T) / (np.pi * T) ** 1.5
        f.append(np.stack([m * (1 + 0.02 * rng.uniform(-1, 1, m.shape))
                           for _ in range(3)]))
    alpha, omega = 1.4, 0.81
    gam = np.full((2, 2), 2 * (1 - omega))
    eta = np.full((2, 2), alpha - 1)
    pre = np.array([[0.1, 0.11], [0.12, 0.13]])
    op = VSSOperator(N, vm.L, vm.qz, vm.qw, vm.sz, vm.sw, szpre, masses, gam,
                     eta, pre, max_evals=2, precision=precision)
    fd = [torch.tensor(x, device='cuda') for x in f]
    src = torch.tensor([2, 0, 1], dtype=torch.int32, device='cuda')
    dst = torch.tensor([0, 2, 1], dtype=torch.int32, device='cuda')
    tol = FP64_TOL if precision == 'fp64' else FP32_TOL
    tabs = {}
    for p in range(2):
        Q0 = torch.randn_like(fd[p]) * 1e-6
        Q = Q0.clone()
        op.eval_species(p, fd, Q, src=src, dst=dst)
        torch.cuda.synchronize()
        got = (Q - Q0).cpu().numpy()
        for s, d in zip(src.tolist(), dst.tolist()):
            ref = np.zeros(N ** 3)
            for q in range(2):
                key = masses[q] / (masses[p] + masses[q])
                if key not in tabs:
                    tabs[key] = oc.VSSTables(N, vm.L, vm.qz, vm.qw, vm.sz, vm.sw,
                                             szpre, gam[p, q], eta[p, q], key)
                ref += oc.vss_fs(tabs[key], pre[p, q], masses[p], masses[q],
                                 f[p][s], f[q][s])
            err = _rel(got[d], ref)
            assert err < tol, (N, p, s, precision, err)
