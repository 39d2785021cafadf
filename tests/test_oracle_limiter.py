"""The oracle's linear slope limiter (dgfsABstd1D ``[time-integrator]
limiter = 1``) against golden vectors from the reference: its basis'
operators (basis.py:289-301) and its limitLin kernel (astd/kernels/
limiters.mako:17-76), compiled for the CPU."""
import os

import numpy as np

from oracle import dg as odg

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def test_limiter_matches_reference():
    z = np.load(os.path.join(G, 'limiter_N4.npz'))
    K, Ne = int(z['K']), int(z['Ne'])
    b = odg.NodalBasis('nodal-sem-gll', K, K)
    assert np.array_equal(b.cellAvgOp, z['Aavg'])
    assert np.array_equal(b.drLinOp, z['Adr'])
    u = z['u'].reshape(K, Ne, -1)
    out = odg.limit_linear(b, z['invjac'], z['xsol'], u)
    assert np.array_equal(out.ravel(), z['ulim'])
    # the limiter is active on this profile and keeps every cell average
    assert np.mean(out.ravel() != u.ravel()) > 0.3
    avg = lambda x: np.einsum('kj,jev->kev', b.cellAvgOp, x)[0]
    assert np.allclose(avg(out), avg(u), rtol=1e-13, atol=0)


def test_package_basis_limiter_operators():
    from dgfs1d_gpu_b200.basis import get_basis
    from dgfs1d_gpu_b200.config import Config
    from dgfs1d_gpu_b200.configs import couette_std_ini
    z = np.load(os.path.join(G, 'limiter_N4.npz'))
    b = get_basis(Config(couette_std_ini()))
    assert np.array_equal(b.cellAvgOp, z['Aavg'])
    assert np.array_equal(b.drLinOp, z['Adr'])
