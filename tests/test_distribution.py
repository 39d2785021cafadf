"""Checkpoint files of the distribution writer (CPU): the datasets and
attributes of std/distribution.py and bi/distribution.py, the file-name
pattern, and the K / Ne / Nv checks of a restart."""
import numpy as np
import pytest

from dgfs1d_gpu_b200.config import Config
from dgfs1d_gpu_b200.distribution import (DGFSDistributionWriter,
                                          read_distribution, remaining_steps,
                                          write_distribution)


class _T:
    """Stands in for a device tensor (the writer calls .detach().cpu())."""

    def __init__(self, a):
        self.a = a

    def detach(self):
        return self

    def cpu(self):
        return self

    def numpy(self):
        return self.a


def test_round_trip_and_checks(tmp_path):
    rng = np.random.default_rng(5)
    a, b = rng.standard_normal(3 * 4 * 8), rng.standard_normal(3 * 4 * 8)
    p = str(tmp_path / 'x.npz_rank=0')
    write_distribution(p, {'coeff0': a, 'coeff1': b}, 0.125, 3, 4, 8)
    got, t = read_distribution(p, ['coeff0', 'coeff1'], 3, 4, 8)
    assert t == 0.125
    assert np.array_equal(got['coeff0'], a) and np.array_equal(got['coeff1'], b)
    for K, Ne, Nv, what in ((2, 4, 8, 'K'), (3, 5, 8, 'Ne'), (3, 4, 9, 'N')):
        with pytest.raises(ValueError, match='Inconsistent distribution ' + what):
            read_distribution(p, ['coeff0'], K, Ne, Nv)
    with pytest.raises(KeyError):
        read_distribution(p, ['coeff'], 3, 4, 8)


def test_writer_schedule_and_names(tmp_path):
    cfg = Config('[dgfsdistwriter]\nbasedir = %s\nbasename = d-{t:.3f}\n'
                 'dt-out = 0.5\n' % tmp_path)
    w = DGFSDistributionWriter(0.0, (3, 2, 8), cfg)
    u = _T(np.arange(48.0))
    assert w(0.25, 0.25, u) is None                 # not an output time
    p = w(0.25, 0.5, u)
    assert p.endswith('d-0.500.npz_rank=0')
    got, t = read_distribution(p, ['coeff'], 3, 2, 8)
    assert t == 0.5 and np.array_equal(got['coeff'], np.arange(48.0))
    assert w(0.25, 0.75, u) is None and w(0.25, 1.0, u) is not None
    wb = DGFSDistributionWriter(0.0, (3, 2, 8), cfg, nspcs=2)
    p = wb(0.5, 0.5, [u, _T(2 * np.arange(48.0))])
    got, _ = read_distribution(p, ['coeff0', 'coeff1'], 3, 2, 8)
    assert np.array_equal(got['coeff1'], 2 * np.arange(48.0))
    off = DGFSDistributionWriter(0.0, (3, 2, 8), Config('[x]\na = 1\n'))
    assert off(0.5, 0.5, u) is None


def test_remaining_steps():
    assert remaining_steps(0.0, 1.0, 0.25) == 4
    assert remaining_steps(0.5, 1.0, 0.25) == 2
    assert remaining_steps(0.1 + 0.2, 0.3, 0.1) == 0
    assert remaining_steps(1.0, 1.0, 0.1) == 0


def test_command_line_parsing(tmp_path):
    """``python -m dgfs1d_gpu_b200 <driver> run|restart ini [dist] -v s::k v``
    (the reference's console-script interface) parses and applies overrides."""
    from dgfs1d_gpu_b200.__main__ import parse
    from dgfs1d_gpu_b200.configs import couette_std_ini
    ini = tmp_path / 'c.ini'
    ini.write_text(couette_std_ini())
    a = parse(['dgfsStd1D', 'run', str(ini), '-v', 'mesh::Ne', '6',
               '-v', 'time-integrator::scheme', 'ssp-rk2'])
    cfg = Config.load(a.inp, defaults=Config.overrides(a.v))
    assert cfg.lookupint('mesh', 'Ne') == 6
    assert cfg.lookup('time-integrator', 'scheme') == 'ssp-rk2'
    b = parse(['dgfsABUstd1D', 'restart', str(ini), 'd.npz_rank=0'])
    assert b.cmd == 'restart' and b.dist == ['d.npz_rank=0']
    with pytest.raises(SystemExit):
        parse(['dgfsNope1D', 'run', str(ini)])


def test_grid_convergence_error(tmp_path):
    """dgfsStdError1D on two checkpoints (Ne and 2 Ne elements): zero for a
    polynomial the nodal basis holds exactly, the restated L1 norm for a
    non-polynomial profile, and the element-count check."""
    from dgfs1d_gpu_b200.error import compute_error
    from dgfs1d_gpu_b200.quadrature import gauss_lobatto_jacobi, lagrange_at
    K, Nv = 3, 5
    z, w = gauss_lobatto_jacobi(K)

    def field(Ne, fn):
        x = np.linspace(0, 1, Ne + 1)
        xs = np.array([0.5 * (x[j] + x[j + 1]) + 0.5 * (x[j + 1] - x[j]) * z
                       for j in range(Ne)]).T                   # (K, Ne)
        amp = np.arange(1, Nv + 1, dtype=float)
        return fn(xs)[:, :, None] * amp[None, None, :]

    def save(name, u):
        p = str(tmp_path / name)
        write_distribution(p, {'coeff': u.ravel()}, 0.0, K, u.shape[1], Nv)
        return p
    quad = lambda x: 1 + x - 2 * x ** 2
    assert compute_error(save('a', field(4, quad)), save('b', field(8, quad))) < 1e-15
    f = lambda x: np.sin(3 * x)
    u1, u2 = field(4, f), field(8, f)
    err = compute_error(save('c', u1), save('d', u2))
    # restated: coarse interpolant at the fine nodes vs the fine values
    r2 = np.concatenate((-np.flip(z * 0.5 + 0.5), z * 0.5 + 0.5))
    im = lagrange_at(z, r2)
    ref = 0.0
    for j in range(4):
        fine = np.concatenate((u2[:, 2 * j], u2[:, 2 * j + 1]), axis=0)  # (2K, Nv)
        d = np.abs(im @ u1[:, j] - fine)
        ref += 0.5 * (w @ d[:K]).sum() + 0.5 * (w @ d[K:]).sum()
    assert err > 0 and abs(err - ref / 8 / Nv) < 1e-15
    with pytest.raises(ValueError, match='2 \\*'):
        compute_error(save('e', u1), save('f', field(12, f)))


def test_nan_check():
    """[dgfsnancheck] nsteps: a NaN in any solution array raises at the
    checked steps only (CPU tensors; the drivers pass their device arrays)."""
    import torch
    from dgfs1d_gpu_b200.nancheck import DGFSNaNCheck
    chk = DGFSNaNCheck(Config('[dgfsnancheck]\nnsteps = 2\n'))
    good, bad = torch.ones(4), torch.tensor([1.0, float('nan')])
    chk(0.1, 1, [good, bad])                       # not a checked step
    chk(0.2, 2, [good])
    with pytest.raises(RuntimeError, match='NaNs detected at t = 0.2'):
        chk(0.2, 2, [good, bad])
    DGFSNaNCheck(Config('[x]\na = 1\n'))(0.0, 2, [bad])   # section absent: off
