"""Oracle restatement of the penalised IMEX path of dgfsABstd1D (float64).

Test infrastructure only (see ``oracle/__init__.py``).  Kernels restate
dgfs1D/astd/kernels/scattering/bgk-direct-gll.mako (cmaxwellian :118-153,
collide :157-181, updateMom{q}_BDF :16-42, updateDistribution{q}_BDF
:46-78, updateMom{q}_LM :327-351, updateDistribution{q}_LM :354-405); the
schemes restate dgfs1D/astd/integrator.py (ARS :56-179 and SSPL :182-278
for the BGK model without Boltzmann operator, bdf-111 :281-322, bdf-222
:325-400, bdf-333 :401-488, boltz-ars-111 :491-552, IMEX-LM :623-792).  Start-up steps of the multi-step schemes use
first-order substeps of the same family (the reference uses ARS-222/443
substeps); ``imex-lm-*`` does not stop after its first step (astd/
integrator.py:732 exits the process there).

The ES-BGK and Shakov penalty models restate esbgk-direct-gll.mako (momentNorm
:157-217, cmaxwellian :220-254, updateMom{q}_BDF :16-81, updateMom{q}_LM
:480-540) and shakov-direct-gll.mako (momentNorm :193-235, cmaxwellian
:237-278, updateMom{q}_BDF :18-120, updateMom{q}_LM :549-645); their
distribution updates and collide are the BGK ones with the model's Gaussian.
"""
import numpy as np


def moments5(f, cv, cw):
    """(npts, 5): rho, rho u, E = sum f |c|^2 cw (astd/scattering.py:155-162)."""
    phi = np.vstack([np.ones(cv.shape[1]), cv, np.sum(cv * cv, axis=0)]) * cw
    return f.reshape(-1, cv.shape[1]) @ phi.T


def temperature(U):
    return (U[:, 4] - (U[:, 1] ** 2 + U[:, 2] ** 2 + U[:, 3] ** 2) / U[:, 0]) \
        / (1.5 * U[:, 0])


def maxwellian(U, cv):
    T = temperature(U)[:, None]
    u = U[:, 1:4] / U[:, 0:1]
    d2 = sum((cv[i][None, :] - u[:, i:i + 1]) ** 2 for i in range(3))
    return U[:, 0:1] / (np.pi * T) ** 1.5 * np.exp(-d2 / T)


def nu(U, prefac, omega):
    return prefac * U[:, 0] * temperature(U) ** (1. - omega)


def collide(U, f, cv, prefac, omega):
    M = maxwellian(U, cv)
    return nu(U, prefac, omega)[:, None] * (M - f.reshape(M.shape))


def implicit(U, rhs, cv, adiv, cdt, prefac, omega):
    """f = (rhs + cdt nu M)/(adiv + cdt nu)."""
    M = maxwellian(U, cv)
    n = nu(U, prefac, omega)[:, None]
    return (rhs.reshape(M.shape) + cdt * n * M) / (adiv + cdt * n)


def moment_rows(cv, nalph):
    """Rows (1, c, |c|^2, c_x^2, c_y^2, c_z^2, c_x c_y, c_y c_z, c_z c_x,
    |c|^2 c) of the penalty models' moment matrix, the first nalph
    (astd/scattering.py:155-162, 306-316, 375-388)."""
    c2 = np.sum(cv * cv, axis=0)
    rows = [np.ones(cv.shape[1]), cv[0], cv[1], cv[2], c2, cv[0] ** 2,
            cv[1] ** 2, cv[2] ** 2, cv[0] * cv[1], cv[1] * cv[2],
            cv[2] * cv[0], c2 * cv[0], c2 * cv[1], c2 * cv[2]]
    return np.vstack(rows[:nalph])


def moments_n(f, cv, cw, nalph):
    return f.reshape(-1, cv.shape[1]) @ (moment_rows(cv, nalph) * cw).T


# stress pairs (i, j) of moments 8, 9, 10 and the stress rows entering the
# heat-flux components: x (5, 8, 10), y (8, 6, 9), z (10, 9, 7)
_OFF = [(1, 2), (2, 3), (3, 1)]
_QROW = [(5, 8, 10), (8, 6, 9), (10, 9, 7)]


class BGKModel:
    nalph = 5

    def __init__(self, Pr=1.0):
        self.Pr = Pr

    def gaussian(self, U, cv):
        return maxwellian(U[:, :5], cv)

    def relax(self, U, adiv, cdt, prefac, omega):
        return U.copy()


class ESBGKModel(BGKModel):
    """Anisotropic Gaussian with T_ij = T/Pr delta_ij + 2(1 - 1/Pr)(P_ij/rho
    - u_i u_j); the stress moments relax with rate nu/Pr."""
    nalph = 11

    def __init__(self, Pr=2. / 3.):
        self.Pr = Pr

    def gaussian(self, U, cv):
        rho = U[:, 0]
        u = U[:, 1:4] / rho[:, None]
        T = U[:, 4] / (1.5 * rho) - np.sum(u * u, axis=1) / 1.5
        lam, mu = 1. / self.Pr, 2. * (1. - 1. / self.Pr)
        A = np.zeros((U.shape[0], 3, 3))
        for i in range(3):
            A[:, i, i] = lam * T + mu * (U[:, 5 + i] / rho - u[:, i] ** 2)
        for k, (i, j) in enumerate(_OFF):
            v = mu * (U[:, 8 + k] / rho - u[:, i - 1] * u[:, j - 1])
            A[:, i - 1, j - 1] = A[:, j - 1, i - 1] = v
        det = np.linalg.det(A)
        Ainv = np.linalg.inv(A)
        d = cv[None, :, :] - u[:, :, None]            # (npts, 3, nv)
        q = np.einsum('pin,pij,pjn->pn', d, Ainv, d)
        return rho[:, None] / (np.pi ** 1.5 * np.sqrt(det)[:, None]) * np.exp(-q)

    def relax(self, U, adiv, cdt, prefac, omega):
        V = U.copy()
        rho, T = U[:, 0], temperature(U[:, :5])
        k = cdt / self.Pr * prefac * rho * T ** (1. - omega)
        for s in (5, 6, 7):
            tau = 0.5 * rho * T + U[:, s - 4] ** 2 / rho
            V[:, s] = (adiv * U[:, s] + k * tau) / (adiv + k)
        for n, (i, j) in enumerate(_OFF):
            tau = U[:, i] * U[:, j] / rho
            V[:, 8 + n] = (adiv * U[:, 8 + n] + k * tau) / (adiv + k)
        return V


class ShakovModel(BGKModel):
    """Maxwellian times 1 + 2(1 - Pr)/5 (q.d)/(rho T^2) (2|d|^2/T - 5) with
    the peculiar heat flux q; stresses relax with rate nu, the heat flux with
    rate Pr nu."""
    nalph = 14

    def __init__(self, Pr=2. / 3.):
        self.Pr = Pr

    def heat_flux(self, U):
        rho = U[:, 0]
        u = U[:, 1:4] / rho[:, None]
        T = U[:, 4] / (1.5 * rho) - np.sum(u * u, axis=1) / 1.5
        u2 = np.sum(u * u, axis=1)
        q = np.empty((U.shape[0], 3))
        for i, (a, b, c) in enumerate(_QROW):
            q[:, i] = (U[:, 11 + i] - 2 * (U[:, a] * u[:, 0] + U[:, b] * u[:, 1]
                                           + U[:, c] * u[:, 2])
                       + rho * u[:, i] * u2 - 1.5 * u[:, i] * rho * T)
        return rho, u, T, q

    def gaussian(self, U, cv):
        rho, u, T, q = self.heat_flux(U)
        d = cv[None, :, :] - u[:, :, None]
        d2 = np.sum(d * d, axis=1)
        M = rho[:, None] / (np.pi * T[:, None]) ** 1.5 * np.exp(-d2 / T[:, None])
        qd = np.einsum('pi,pin->pn', q, d)
        return M * (1. + 2. * (1. - self.Pr) / 5. * qd
                    / (rho * T * T)[:, None] * (2. * d2 / T[:, None] - 5.))

    def relax(self, U, adiv, cdt, prefac, omega):
        V = U.copy()
        rho, T = U[:, 0], temperature(U[:, :5])
        nu_ = prefac * rho * T ** (1. - omega)
        k = cdt * nu_
        for s in (5, 6, 7):
            tau = 0.5 * rho * T + U[:, s - 4] ** 2 / rho
            V[:, s] = (adiv * U[:, s] + k * tau) / (adiv + k)
        for n, (i, j) in enumerate(_OFF):
            tau = U[:, i] * U[:, j] / rho
            V[:, 8 + n] = (adiv * U[:, 8 + n] + k * tau) / (adiv + k)
        m2 = np.sum(U[:, 1:4] ** 2, axis=1) / rho ** 2
        Pr = self.Pr
        for i, (a, b, c) in enumerate(_QROW):
            ru = U[:, 1 + i]
            tq = ((1. - Pr) * (-2. * (V[:, a] * U[:, 1] + V[:, b] * U[:, 2]
                                      + V[:, c] * U[:, 3]) / rho
                               + ru * m2 - 1.5 * ru * T)
                  + (ru * m2 + 2.5 * ru * T))
            V[:, 11 + i] = (adiv * U[:, 11 + i] + k * tq) / (adiv + Pr * k)
        return V


def model_collide(model, U, f, cv, prefac, omega):
    M = model.gaussian(U, cv)
    return nu(U[:, :5], prefac, omega)[:, None] * (M - f.reshape(M.shape))


def model_implicit(model, U, rhs, cv, adiv, cdt, prefac, omega):
    """f = (rhs + cdt nu G(U))/(adiv + cdt nu) with the model's Gaussian."""
    M = model.gaussian(U, cv)
    n = nu(U[:, :5], prefac, omega)[:, None]
    return (rhs.reshape(M.shape) + cdt * n * M) / (adiv + cdt * n)


# (A, B, C) of the IMEX linear multistep schemes, astd/integrator.py:736-907
BDF_COEF = {
    'bdf-222': ([1. / 3., -4. / 3., 1.], [-2. / 3., 4. / 3.], 2. / 3.),
    'bdf-333': ([-2. / 11., 9. / 11., -18. / 11., 1.], [6. / 11., -18. / 11., 18. / 11.],
                6. / 11.),
}

# ARS (astd/integrator.py:117-179) and SSPL (:240-278) tables: (_A, A) and,
# for SSPL, the weights (_w, w)
_g2 = 1. - (2. ** 0.5) / 2.
_d2 = 1. - 1. / (2. * _g2)
ARS_COEF = {
    'ars-111': ([[0., 0.], [1., 0.]], [[0., 0.], [0., 1.]]),
    'ars-222': ([[0., 0., 0.], [_g2, 0., 0.], [_d2, 1 - _d2, 0.]],
                [[0., 0., 0.], [0., _g2, 0.], [0., 1 - _g2, _g2]]),
    'ars-443': ([[0., 0., 0., 0., 0.], [1. / 2., 0., 0., 0., 0.],
                 [11. / 18., 1. / 18., 0., 0., 0.], [5. / 6., -5. / 6., 1. / 2., 0., 0.],
                 [1. / 4., 7. / 4., 3. / 4., -7. / 4., 0.]],
                [[0., 0., 0., 0., 0.], [0., 1. / 2., 0., 0., 0.], [0., 1. / 6., 1. / 2., 0., 0.],
                 [0., -1. / 2., 1. / 2., 1. / 2., 0.], [0., 3. / 2., -3. / 2., 1. / 2., 1. / 2.]]),
}
_al, _be, _et = 0.24169426078821, 0.06042356519705, 0.12915286960590
SSPL_COEF = {
    'sspl-222': ([[0., 0.], [1., 0.]], [[_g2, 0.], [1 - 2 * _g2, _g2]],
                 [0.5, 0.5], [0.5, 0.5]),
    'sspl-443': ([[0., 0., 0., 0.], [0., 0., 0., 0.], [0., 1., 0., 0.],
                  [0., 1. / 4., 1. / 4., 0.]],
                 [[_al, 0., 0., 0.], [-_al, _al, 0., 0.], [0., 1. - _al, _al, 0.],
                  [_be, _et, 1. / 2. - _be - _et - _al, _al]],
                 [0., 1. / 6., 1. / 6., 2. / 3.], [0., 1. / 6., 1. / 6., 2. / 3.]),
}

LM_COEF = {
    'imex-lm-bdf1': ([-1.], [1.], [1., 0.]),
    'imex-lm-bdf2': ([-4. / 3., 1. / 3.], [4. / 3., -2. / 3.], [2. / 3., 0., 0.]),
    'imex-lm-cn2': ([-1., 0.], [1.5, -0.5], [0.5, 0.5, 0.]),
    'imex-lm-ad2': ([-1., 0.], [1.5, -0.5], [9. / 16., 3. / 8., 1. / 16.]),
    'imex-lm-sg2': ([-3. / 4., 0., -1. / 4.], [3. / 2., 0., 0.], [1., 0., 0., 1. / 2.]),
    'imex-lm-bdf3': ([-18. / 11., 9. / 11., -2. / 11.], [18. / 11., -18. / 11., 6. / 11.],
                     [6. / 11., 0., 0., 0.]),
    'imex-lm-ad3': ([-1., 0., 0.], [23. / 12., -4. / 3., 5. / 12.],
                    [4661. / 10000., 15551. / 30000., 1949. / 30000., -1483. / 30000.]),
    'imex-lm-tvb3': ([-3909. / 2048., 1367. / 1024., -873. / 2048.],
                     [18463. / 12288., -1271. / 768., 8233. / 12288.],
                     [1089. / 2048., -1139. / 12288., -367. / 6144., 1699. / 12288.]),
    'imex-lm-bdf4': ([-48. / 25., 36. / 25., -16. / 25., 3. / 25.],
                     [48. / 25., -72. / 25., 48. / 25., -12. / 25.],
                     [12. / 25., 0., 0., 0., 0.]),
    'imex-lm-tvb4': ([-21531. / 8192., 22753. / 8192., -12245. / 8192., 2831. / 8192.],
                     [13261. / 8192., -75029. / 24576., 54799. / 24576., -15245. / 24576.],
                     [4207. / 8192., -3567. / 8192., 697. / 24576., 4315. / 24576.,
                      -41. / 384.]),
    'imex-lm-shu3': ([-16. / 27, 0., 0., -11. / 27.], [16. / 9., 0., 0., 4. / 9.],
                     [9035. / 19683., 13541. / 19683., 1127. / 2187., 7927. / 19683.,
                      3094. / 19683.]),
    'imex-lm-shu4': ([-137. / 400., 0., 0., -959. / 5000., -8781. / 94000.,
                      -87487 / 235000.],
                     [976903. / 470000., 0., 0., 136757. / 117500., 266997. / 470000., 0.],
                     [237. / 500., 7547. / 10000., 299. / 400., 4513. / 5875.,
                      118099. / 235000., 174527. / 470000., 90349. / 470000.]),
}


class IMEX:
    """Penalised schemes on (K, Ne, Nv) arrays.

    explicit(f) -> DG advection; boltz(f) -> Q(f) or None (BGK only).
    """

    def __init__(self, kind, explicit, boltz, cv, cw, prefac, omega, dt,
                 f0, nsub=10, model=None):
        self.kind, self.cv, self.cw = kind, cv, cw
        self.prefac, self.omega, self.dt = prefac, omega, dt
        self.explicit, self.boltz = explicit, boltz
        self.model = model if model is not None else BGKModel()
        self.shape = f0.shape
        self.step_no = 0
        self.starts = []
        if kind in BDF_COEF:
            k = len(BDF_COEF[kind][1])
            f = f0.copy()
            helper = IMEX('bdf-111', explicit, boltz, cv, cw, prefac, omega,
                          dt / nsub, f0, model=self.model)
            self.hist = [self._bdf_state(f0)]
            for _ in range(k - 1):
                for _ in range(nsub):
                    f = helper.step(f)
                self.starts.append(f.copy())
                self.hist.append(self._bdf_state(f))
        elif kind in LM_COEF:
            s = len(LM_COEF[kind][0])
            self.hist = [self._state(f0)]
            if s > 1:
                f = f0.copy()
                helper = IMEX('imex-lm-bdf1', explicit, boltz, cv, cw, prefac,
                              omega, dt / nsub, f0, model=self.model)
                for _ in range(1, s):
                    for _ in range(nsub):
                        f = helper.step(f)
                    self.starts.append(f.copy())
                    self.hist.append(self._state(f))

    def _mom(self, x):
        return moments_n(x, self.cv, self.cw, self.model.nalph)

    def _implicit(self, U, rhs, adiv, cdt):
        return model_implicit(self.model, U, rhs, self.cv, adiv, cdt,
                              self.prefac, self.omega).reshape(self.shape)

    def _collide(self, U, f):
        return model_collide(self.model, U, f, self.cv, self.prefac,
                             self.omega).reshape(self.shape)

    def _relax(self, U, adiv, cdt):
        return self.model.relax(U, adiv, cdt, self.prefac, self.omega)

    def _state(self, f):
        U = self._mom(f)
        P = self._collide(U, f)
        E = self.explicit(f) + self.boltz(f) - P
        return dict(F=f.copy(), U=U, P=P, LM=self._mom(P), L=E,
                    LU=self._mom(E))

    def _bdf_state(self, f):
        L = self.explicit(f)
        return dict(F=f.copy(), U=self._mom(f), L=L, LU=self._mom(L))

    def _ars_stage(self, F0, Ls, Ps, ex, im, aqq, U):
        # updateDistribution{q}_ARS (bgk-direct-gll.mako:233-279): the
        # explicit sum over the stage advections, the implicit sum over the
        # earlier stages' penalties and the implicit last stage
        dt = self.dt
        rhs = F0 + sum(a * dt * L for a, L in zip(ex, Ls)) + \
            sum(a * dt * P for a, P in zip(im, Ps))
        return self._implicit(U, rhs, 1., aqq * dt)

    def step(self, f):
        dt, k = self.dt, self.kind
        if k in ARS_COEF:
            # ARSabcIntegratorAstd._integrate (astd/integrator.py:56-114)
            _A, A = ARS_COEF[k]
            ns = len(A) - 1
            U0 = self._mom(f)
            Fs, Ls, LUs, Ps = [f], [], [], []
            for i in range(ns):
                Ls.append(self.explicit(Fs[i]))
                LUs.append(self._mom(Ls[i]))
                ex = _A[i + 1][:i + 1]
                U = U0 + sum(dt * a * LU for a, LU in zip(ex, LUs))
                Fq = self._ars_stage(f, Ls, Ps, ex, A[i + 1][1:i + 1],
                                     A[i + 1][i + 1], U)
                Fs.append(Fq)
                Ps.append(self._collide(U, Fq))
            return Fs[-1]
        if k in SSPL_COEF:
            # SSPLabcIntegratorAstd._integrate (astd/integrator.py:182-228)
            _A, A, _w, w = SSPL_COEF[k]
            ns = len(A)
            U0 = self._mom(f)
            F1 = self._ars_stage(f, [], [], [], [], A[0][0], U0)
            Fs, Ls, LUs, Ps = [f, F1], [], [], [self._collide(U0, F1)]
            for i in range(1, ns):
                Ls.append(self.explicit(Fs[i]))
                LUs.append(self._mom(Ls[-1]))
                ex = _A[i][:i]
                U = U0 + sum(dt * a * LU for a, LU in zip(ex, LUs))
                Fq = self._ars_stage(f, Ls, Ps, ex, A[i][:i], A[i][i], U)
                Fs.append(Fq)
                Ps.append(self._collide(U, Fq))
            Ls.append(self.explicit(Fs[ns]))
            # updateDistributionWeight{q}_SSPL (bgk-direct-gll.mako:282-326)
            return f + sum(a * dt * L for a, L in zip(_w, Ls)) + \
                sum(a * dt * P for a, P in zip(w, Ps))
        if k == 'boltz-ars-111':
            # integrator.py:491-552: moments of the advection only, then the
            # explicit part L + Q - P (P = nu (M(U0) - f)) in the update of f
            U0 = self._mom(f)
            P0 = self._collide(U0, f)
            L0 = self.explicit(f)
            LU0 = self._mom(L0)
            L0 = L0 + self.boltz(f) - P0
            U = self._relax(-((-1.) * U0 + (-1.) * dt * LU0) / 1., 1., dt)
            rhs = -((-1.) * f + (-1.) * dt * L0)
            return self._implicit(U, rhs, 1., dt)
        if k == 'bdf-111':
            U0 = self._mom(f)
            L0 = self.explicit(f)
            LU0 = self._mom(L0)
            U = self._relax(-((-1.) * U0 + (-1.) * dt * LU0) / 1., 1., dt)
            rhs = -((-1.) * f + (-1.) * dt * L0)
            return self._implicit(U, rhs, 1., dt)
        if k in BDF_COEF:
            # integrator.py:325-488 (updateMom{q}_BDF, updateDistribution{q}_BDF)
            A, G, b = BDF_COEF[k]
            q = len(G)
            if self.step_no < q - 1:
                self.step_no += 1
                return self.starts[self.step_no - 1].copy()
            hs = self.hist
            U = -sum(A[i] * hs[i]['U'] + (-G[i]) * dt * hs[i]['LU']
                     for i in range(q)) / A[q]
            U = self._relax(U, A[q], b * dt)
            rhs = -sum(A[i] * hs[i]['F'] + (-G[i]) * dt * hs[i]['L']
                       for i in range(q))
            fn = self._implicit(U, rhs, A[q], b * dt)
            self.hist = hs[1:] + [self._bdf_state(fn)]
            self.step_no += 1
            return fn
        if k in LM_COEF:
            A, B, C = LM_COEF[k]
            s = len(A)
            if s > 1 and self.step_no < s - 1:
                self.step_no += 1
                return self.starts[self.step_no - 1].copy()
            hs = self.hist
            U = sum(-A[s - i - 1] * hs[i]['U'] + dt * B[s - i - 1] * hs[i]['LU']
                    + dt * C[s - i] * hs[i]['LM'] for i in range(s))
            rhs = sum(-A[s - i - 1] * hs[i]['F'] + dt * B[s - i - 1] * hs[i]['L']
                      + dt * C[s - i] * hs[i]['P'] for i in range(s))
            U = self._relax(U, 1., C[0] * dt)
            fn = self._implicit(U, rhs, 1., C[0] * dt)
            P = self._collide(U, fn)
            E = self.explicit(fn) + self.boltz(fn) - P
            new = dict(F=fn.copy(), U=U, P=P, LM=self._mom(P), L=E,
                       LU=self._mom(E))
            self.hist = hs[1:] + [new]
            self.step_no += 1
            return fn
        raise ValueError(k)


def std_esbgk_relax(f, cv, cw, prefac, omega, Pr):
    """Explicit ES-BGK relaxation of dgfsStd1D (esbgk-direct-gll fs,
    std/scattering.py:1540-1637 with std/kernels/scattering/esbgk-direct-gll.mako):
    Q = prefac rho / T^(omega-1) (f_ES - f), f_ES the Gaussian whose covariance
    is the discrete second moment of (1-1/Pr) f + (1/Pr) f_M normalised by rho
    (f_M the grid Maxwellian).  f: (Nv,)."""
    s0 = f.sum()
    u = np.array([(f * cv[i]).sum() / s0 for i in range(3)])
    rho = s0 * cw
    d = cv - u[:, None]
    T = (f * (d * d).sum(axis=0)).sum() * (cw / (1.5 * rho))
    fm = rho / (np.pi * T) ** 1.5 * np.exp(-(d * d).sum(axis=0) / T)
    w = (1. - 1. / Pr) * f + (1. / Pr) * fm
    S = np.array([[(d[i] * d[j] * w).sum() for j in range(3)] for i in range(3)]) * cw / rho
    A = np.linalg.inv(S)
    q = np.einsum('iv,ij,jv->v', d, A, d)
    fes = rho / ((2 * np.pi) ** 1.5 * np.sqrt(np.linalg.det(S))) * np.exp(-q / 2.)
    return prefac * (rho / T ** (omega - 1.)) * (fes - f)
