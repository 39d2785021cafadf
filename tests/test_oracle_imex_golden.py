"""The IMEX oracle's kernels against the reference's bgk-direct-gll.mako,
esbgk-direct-gll.mako and shakov-direct-gll.mako."""
import os

import numpy as np
import pytest

from oracle import imex as oim
from oracle import imex as oi

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b))
                 / np.linalg.norm(np.ravel(b)))


def test_penalty_kernels_match_reference():
    g = np.load(os.path.join(G, 'penalty_N8.npz'))
    npts, cv, cw = int(g['npts']), g['cv'], float(g['cw'])
    f = g['f'].reshape(npts, -1)
    U = oim.moments5(f, cv, cw)
    assert _rel(U, g['U'].reshape(npts, 5)) < 1e-14
    U = g['U'].reshape(npts, 5)
    assert _rel(oim.maxwellian(U, cv), g['M']) < 1e-13
    pre, om = float(g['prefac']), float(g['omega'])
    assert _rel(oim.collide(U, f, cv, pre, om), g['Q']) < 1e-12
    dt = float(g['dt'])
    a1, a2, a3, g1, g2, b = 1. / 3., -4. / 3., 1., -2. / 3., 4. / 3., 2. / 3.
    U0, U1 = U, g['U1'].reshape(npts, 5)
    LU0, LU1 = g['LU0'].reshape(npts, 5), g['LU1'].reshape(npts, 5)
    Un = -(a1 * U0 + (-g1) * dt * LU0 + a2 * U1 + (-g2) * dt * LU1) / a3
    assert _rel(Un, g['Un_bdf2']) < 1e-14
    rhs = -(a1 * g['f'] + (-g1) * dt * g['L0'] + a2 * g['f1'] + (-g2) * dt * g['L1'])
    # the kernel takes the Maxwellian as an argument (the golden passed the
    # one of U0); nu comes from the new moments
    M = g['M'].reshape(npts, -1)
    nu = oim.nu(Un, pre, om)[:, None]
    fn = (rhs.reshape(M.shape) + b * dt * nu * M) / (a3 + b * dt * nu)
    assert _rel(fn, g['fn_bdf2']) < 1e-13
    # and with a consistent Maxwellian the oracle's implicit() is that formula
    Mn = oim.maxwellian(Un, cv)
    assert _rel(oim.implicit(Un, rhs, cv, a3, b * dt, pre, om),
                (rhs.reshape(M.shape) + b * dt * nu * Mn) / (a3 + b * dt * nu)) < 1e-15
    A, B, C = [-4. / 3., 1. / 3.], [4. / 3., -2. / 3.], [2. / 3., 0., 0.]
    hs = [dict(U=U0, LU=LU0, LM=g['LM0'].reshape(npts, 5), F=g['f'],
               L=g['L0'], P=g['P0']),
          dict(U=U1, LU=LU1, LM=g['LM1'].reshape(npts, 5), F=g['f1'],
               L=g['L1'], P=g['P1'])]
    s = 2
    U2 = sum(-A[s - i - 1] * hs[i]['U'] + dt * B[s - i - 1] * hs[i]['LU']
             + dt * C[s - i] * hs[i]['LM'] for i in range(s))
    assert _rel(U2, g['U2_lm2']) < 1e-14
    rhs = sum(-A[s - i - 1] * hs[i]['F'] + dt * B[s - i - 1] * hs[i]['L']
              + dt * C[s - i] * hs[i]['P'] for i in range(s))
    nu2 = oim.nu(U2, pre, om)[:, None]
    f2 = (rhs.reshape(M.shape) + C[0] * dt * nu2 * M) / (1.0 + C[0] * dt * nu2)
    assert _rel(f2, g['f2_lm2']) < 1e-13


def test_ars_sspl_stage_matches_reference():
    """One ARS stage and the SSPL weighting of the oracle (the arithmetic of
    IMEX._ars_stage and the SSPL weighted sum) against the reference's
    updateMom2_ARS, updateDistribution2_ARS and updateDistributionWeight2_SSPL
    kernels on the golden data."""
    g = np.load(os.path.join(G, 'penalty_N8.npz'))
    npts, cv = int(g['npts']), g['cv']
    pre, om, dt = float(g['prefac']), float(g['omega']), float(g['dt'])
    _a, a = list(g['ars_a']), list(g['ars_A'])
    U0, U1 = g['U'].reshape(npts, 5), g['U1'].reshape(npts, 5)
    LU0, LU1 = g['LU0'].reshape(npts, 5), g['LU1'].reshape(npts, 5)
    U2 = U0 + dt * _a[0] * LU0 + dt * _a[1] * LU1
    assert _rel(U2, g['U2_ars']) < 1e-14
    assert _rel(oim.maxwellian(U1, cv), g['M1_ars']) < 1e-13
    assert _rel(oim.maxwellian(U2, cv), g['M2_ars']) < 1e-13
    f0, f1 = g['f'].reshape(npts, -1), g['f1'].reshape(npts, -1)
    L0, L1 = g['L0'].reshape(npts, -1), g['L1'].reshape(npts, -1)
    P1 = oim.collide(U1, f1, cv, pre, om)
    rhs = f0 + _a[0] * dt * L0 + _a[1] * dt * L1 + a[0] * dt * P1
    f2 = oim.implicit(U2, rhs, cv, 1.0, a[1] * dt, pre, om)
    assert _rel(f2, g['f2_ars']) < 1e-13
    f2s = g['f2_sspl'].reshape(npts, -1)
    P2 = oim.collide(U2, f2s, cv, pre, om)
    f3 = f0 + 0.5 * dt * L0 + 0.5 * dt * L1 + 0.5 * dt * P1 + 0.5 * dt * P2
    assert _rel(f3, g['f3_sspl']) < 1e-13


@pytest.mark.parametrize('tag', ['esbgk', 'shakov'])
def test_esbgk_shakov_oracle_matches_reference(tag):
    """The oracle's ES-BGK / Shakov penalty models against the reference's
    own kernels (esbgk-direct-gll.mako, shakov-direct-gll.mako compiled for
    the CPU): moments, moment normalisation + Gaussian, collide, and the BDF2
    and IMEX-LM2 moment and distribution updates."""
    z = np.load(os.path.join(G, 'penalty_%s_N8.npz' % tag))
    model = {'esbgk': oi.ESBGKModel, 'shakov': oi.ShakovModel}[tag](float(z['Pr']))
    na, npts, cv, cw = int(z['nalph']), int(z['npts']), z['cv'], float(z['cw'])
    pf, om, dt = float(z['prefac']), float(z['omega']), float(z['dt'])
    f = z['f'].reshape(npts, -1)

    def rel(a, b):
        return float(np.abs(np.ravel(a) - np.ravel(b)).max() / np.abs(np.ravel(b)).max())
    U = oi.moments_n(f, cv, cw, na)
    assert rel(U, z['U']) < 1e-13
    assert rel(model.gaussian(U, cv), z['M']) < 1e-13
    assert rel(oi.model_collide(model, U, f, cv, pf, om), z['Q']) < 1e-12
    sh = lambda k: z[k].reshape(npts, -1)
    a1, a2, a3, g1, g2, b = 1. / 3., -4. / 3., 1., -2. / 3., 4. / 3., 2. / 3.
    Ul = -(a1 * U + (-g1) * dt * sh('LU0') + a2 * sh('U1') + (-g2) * dt * sh('LU1')) / a3
    Un = model.relax(Ul, a3, b * dt, pf, om)
    assert rel(Un, z['Un_bdf2']) < 1e-13
    assert rel(model.gaussian(Un, cv), z['Mn_bdf2']) < 1e-13
    rhs = -(a1 * f + (-g1) * dt * sh('L0') + a2 * sh('f1') + (-g2) * dt * sh('L1'))
    fn = oi.model_implicit(model, Un, rhs, cv, a3, b * dt, pf, om)
    assert rel(fn, z['fn_bdf2']) < 1e-13
    A, B, C = [-4. / 3., 1. / 3.], [4. / 3., -2. / 3.], [2. / 3., 0., 0.]
    Us, LUs, LMs = [U, sh('U1')], [sh('LU0'), sh('LU1')], [sh('LM0'), sh('LM1')]
    Ul = sum(-A[1 - i] * Us[i] + dt * B[1 - i] * LUs[i] + dt * C[2 - i] * LMs[i]
             for i in range(2))
    U2 = model.relax(Ul, 1.0, C[0] * dt, pf, om)
    assert rel(U2, z['U2_lm2']) < 1e-13
    Fs, Ls, Ps = [f, sh('f1')], [sh('L0'), sh('L1')], [sh('P0'), sh('P1')]
    rhs = sum(-A[1 - i] * Fs[i] + dt * B[1 - i] * Ls[i] + dt * C[2 - i] * Ps[i]
              for i in range(2))
    f2 = oi.model_implicit(model, U2, rhs, cv, 1.0, C[0] * dt, pf, om)
    assert rel(f2, z['f2_lm2']) < 1e-13


def test_std_direct_relaxation_matches_reference():
    """dgfsStd1D's explicit bgk-direct-gll / shakov-direct-gll fs (the std
    kernels, golden) equal the penalty models' collide of the oracle."""
    g = np.load(os.path.join(G, 'std_relax_N8.npz'))
    f, cv, cw = g['f'], g['cv'], float(g['cw'])
    pre, om, Pr = float(g['prefac']), float(g['omega']), float(g['Pr'])
    U5 = oim.moments5(f[None], cv, cw)
    assert _rel(oim.collide(U5, f, cv, pre, om).ravel(), g['Q_bgk']) < 1e-12
    U14 = oim.moments_n(f[None], cv, cw, 14)
    Q = oim.model_collide(oim.ShakovModel(Pr), U14, f[None], cv, pre, om).ravel()
    assert _rel(Q, g['Q_shakov']) < 1e-12
    # ES-BGK: the std form (discrete covariance of the grid Maxwellian mix)
    assert _rel(oim.std_esbgk_relax(f, cv, cw, pre, om, Pr), g['Q_esbgk']) < 1e-12
