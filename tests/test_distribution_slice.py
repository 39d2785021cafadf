"""The velocity-slice writer of the single-species driver (CPU tensors):
values against the restated reference slice (std/distributionslice.py:
120-149) and its argument checks."""
import numpy as np
import pytest
import torch

from dgfs1d_gpu_b200.basis import get_basis
from dgfs1d_gpu_b200.config import Config
from dgfs1d_gpu_b200.configs import couette_std_ini
from dgfs1d_gpu_b200.std.distributionslice import DGFSDistributionSliceStd
from dgfs1d_gpu_b200.velocitymesh import DGFSVelocityMeshStd


def _cfg(tmp_path, **keys):
    ini = couette_std_ini(Nv=8, Nrho=4) + '\n[dgfsdistslicewriter]\n'
    ini += 'basedir = %s\nbasename = s-{t:.2f}\ndt-out = 0.5\n' % tmp_path
    ini += ''.join('%s = %s\n' % (k.replace('_', '-'), v) for k, v in keys.items())
    return Config(ini)


@pytest.mark.parametrize('free', ['Nvx_out', 'Nvy_out', 'Nvz_out'])
def test_slice_values_and_file(tmp_path, free):
    keys = dict(Ne_out=2, Nqr_out=1, Nvx_out=1, Nvy_out=5, Nvz_out=6)
    del keys[free]
    cfg = _cfg(tmp_path, **keys)
    vm, basis = DGFSVelocityMeshStd(cfg), get_basis(cfg)
    K, Ne, N = basis.K, 4, vm.Nv()
    rng = np.random.default_rng(3)
    u = rng.standard_normal((K, Ne, N ** 3))
    w = DGFSDistributionSliceStd(0.0, (K, Ne, N ** 3), basis.interpMat, vm, cfg)
    assert w(0.1, 0.25, torch.tensor(u)) is None
    f = w(0.1, 0.5, torch.tensor(u))
    # the reference: interpolate everything, then slice
    sol = np.einsum('mr,mej->rej', basis.interpMat, u)[1, 2].reshape(N, N, N)
    cv = [c.reshape(N, N, N) for c in vm.cv()]
    if free == 'Nvx_out':
        ref, vs = sol[:, 5, 6], cv[0][:, 5, 6]
    elif free == 'Nvy_out':
        ref, vs = sol[1, :, 6], cv[1][1, :, 6]
    else:
        ref, vs = sol[1, 5, :], cv[2][1, 5, :]
    assert np.allclose(f, ref, rtol=1e-14, atol=1e-14)
    data = np.loadtxt(tmp_path / 's-0.50.txt')
    assert np.allclose(data[:, 0], vs) and np.allclose(data[:, 1], ref, rtol=1e-15)


def test_slice_argument_checks(tmp_path):
    def make(**keys):
        cfg = _cfg(tmp_path, **keys)
        vm, basis = DGFSVelocityMeshStd(cfg), get_basis(cfg)
        return DGFSDistributionSliceStd(0.0, (basis.K, 4, vm.Nv() ** 3),
                                        basis.interpMat, vm, cfg)
    with pytest.raises(ValueError, match='2 of the three'):
        make(Ne_out=0, Nqr_out=0)
    with pytest.raises(ValueError, match='Exactly 2'):
        make(Ne_out=0, Nqr_out=0, Nvx_out=1, Nvy_out=1, Nvz_out=1)
    with pytest.raises(ValueError, match='Ne_out'):
        make(Ne_out=4, Nqr_out=0, Nvx_out=1, Nvy_out=1)
    with pytest.raises(ValueError, match='Nqr_out'):
        make(Ne_out=0, Nqr_out=99, Nvx_out=1, Nvy_out=1)
    with pytest.raises(ValueError, match='Nvy-out'):
        make(Ne_out=0, Nqr_out=0, Nvx_out=1, Nvy_out=8)
