"""The oracle's bulk moments against the reference's own moment writers
(golden vectors from DGFSMomWriterStd / DGFSMomWriterBi
``_compute_moments_1D``, std/moments.py:11-70 and bi/moments.py:11-113)."""
import os

import numpy as np

from oracle import dg as odg

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


class _Basis:
    def __init__(self, im):
        self.interpMat = im


def _load():
    return np.load(os.path.join(G, 'moments_N8.npz'))


def test_std_moments_match_reference_writer():
    z = _load()
    got = odg.moments(_Basis(z['interpMat']), z['std_f'], z['std_cv'],
                      float(z['std_cw']), T0=float(z['std_T0']),
                      rho0=float(z['std_rho0']), u0=float(z['std_u0']),
                      molarMass0=float(z['std_molarMass0']))
    ref = z['std_mom']
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max(axis=(0, 1)))


def test_std_moments_zero_density_writes_zeros():
    z = _load()
    got = odg.moments(_Basis(z['interpMat']), 0 * z['std_f'], z['std_cv'],
                      float(z['std_cw']))
    assert np.all(got == 0)


def _bi(z, tag):
    return odg.moments_bi(
        _Basis(z['interpMat']), [z['bi_%s_f0' % tag], z['bi_%s_f1' % tag]],
        z['bi_cv'], float(z['bi_cw']), list(z['bi_masses']),
        T0=float(z['bi_T0']), rho0=float(z['bi_rho0']), u0=float(z['bi_u0']),
        R0=float(z['bi_R0']), NA=float(z['bi_NA']),
        molarMass0=float(z['bi_molarMass0']))


def test_bi_moments_match_reference_writer():
    z = _load()
    for tag in ('mix', 'absent'):
        got, ref = _bi(z, tag), z['bi_%s_mom' % tag]
        scale = np.abs(ref).max(axis=(0, 1))
        assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * scale + 1e-300), tag


def test_bi_absent_species_columns():
    z = _load()
    ref = z['bi_absent_mom']
    assert np.all(ref[:, :, 7:] == 0)          # absent species: all zero
    assert np.all(ref[:, :, 0] > 0)            # present species untouched
