"""Oracle restatement of the penalised IMEX path of dgfsABstd1D (float64).

Test infrastructure only (see ``oracle/__init__.py``).  Kernels restate
dgfs1D/astd/kernels/scattering/bgk-direct-gll.mako (cmaxwellian :118-153,
collide :157-181, updateMom{q}_BDF :16-42, updateDistribution{q}_BDF
:46-78, updateMom{q}_LM :327-351, updateDistribution{q}_LM :354-405); the
schemes restate dgfs1D/astd/integrator.py (bdf-111 :281-322, bdf-222
:325-400, IMEX-LM :623-792).  Start-up steps of the multi-step schemes use
first-order substeps of the same family (the reference uses ARS-222/443
substeps); ``imex-lm-*`` does not stop after its first step (astd/
integrator.py:732 exits the process there).
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


class IMEX:
    """Penalised schemes on (K, Ne, Nv) arrays.

    explicit(f) -> DG advection; boltz(f) -> Q(f) or None (BGK only).
    """

    def __init__(self, kind, explicit, boltz, cv, cw, prefac, omega, dt,
                 f0, nsub=10):
        self.kind, self.cv, self.cw = kind, cv, cw
        self.prefac, self.omega, self.dt = prefac, omega, dt
        self.explicit, self.boltz = explicit, boltz
        self.shape = f0.shape
        self.step_no = 0
        if kind in ('bdf-222', 'imex-lm-bdf2'):
            f = f0.copy()
            sub = 'bdf-111' if kind == 'bdf-222' else 'imex-lm-bdf1'
            helper = IMEX(sub, explicit, boltz, cv, cw, prefac, omega,
                          dt / nsub, f0)
            for _ in range(nsub):
                f = helper.step(f)
            self.start = f
            if kind == 'imex-lm-bdf2':
                self.hist = [self._state(f0), self._state(f)]
            else:
                self.hist = [self._bdf_state(f0), self._bdf_state(f)]
        elif kind == 'imex-lm-bdf1':
            self.hist = [self._state(f0)]

    def _mom(self, x):
        return moments5(x, self.cv, self.cw)

    def _state(self, f):
        U = self._mom(f)
        P = collide(U, f, self.cv, self.prefac, self.omega).reshape(self.shape)
        E = self.explicit(f) + self.boltz(f) - P
        return dict(F=f.copy(), U=U, P=P, LM=self._mom(P), L=E,
                    LU=self._mom(E))

    def _bdf_state(self, f):
        L = self.explicit(f)
        return dict(F=f.copy(), U=self._mom(f), L=L, LU=self._mom(L))

    def step(self, f):
        dt, k = self.dt, self.kind
        if k == 'bdf-111':
            U0 = self._mom(f)
            L0 = self.explicit(f)
            LU0 = self._mom(L0)
            U = -((-1.) * U0 + (-1.) * dt * LU0) / 1.
            rhs = -((-1.) * f + (-1.) * dt * L0)
            return implicit(U, rhs, self.cv, 1., dt, self.prefac,
                            self.omega).reshape(self.shape)
        if k == 'bdf-222':
            a1, a2, a3 = 1. / 3., -4. / 3., 1.
            g1, g2 = -2. / 3., 4. / 3.
            b = 2. / 3.
            if self.step_no == 0:
                self.step_no += 1
                return self.start.copy()
            h0, h1 = self.hist
            U = -(a1 * h0['U'] + (-g1) * dt * h0['LU'] + a2 * h1['U']
                  + (-g2) * dt * h1['LU']) / a3
            rhs = -(a1 * h0['F'] + (-g1) * dt * h0['L'] + a2 * h1['F']
                    + (-g2) * dt * h1['L'])
            fn = implicit(U, rhs, self.cv, a3, b * dt, self.prefac,
                          self.omega).reshape(self.shape)
            self.hist = [h1, self._bdf_state(fn)]
            self.step_no += 1
            return fn
        if k in ('imex-lm-bdf1', 'imex-lm-bdf2'):
            if k == 'imex-lm-bdf1':
                A, B, C = [-1.], [1.], [1., 0.]
            else:
                A, B, C = [-4. / 3., 1. / 3.], [4. / 3., -2. / 3.], [2. / 3., 0., 0.]
            s = len(A)
            if s > 1 and self.step_no < s - 1:
                self.step_no += 1
                return self.start.copy()
            hs = self.hist
            U = sum(-A[s - i - 1] * hs[i]['U'] + dt * B[s - i - 1] * hs[i]['LU']
                    + dt * C[s - i] * hs[i]['LM'] for i in range(s))
            rhs = sum(-A[s - i - 1] * hs[i]['F'] + dt * B[s - i - 1] * hs[i]['L']
                      + dt * C[s - i] * hs[i]['P'] for i in range(s))
            fn = implicit(U, rhs, self.cv, 1., C[0] * dt, self.prefac,
                          self.omega).reshape(self.shape)
            P = collide(U, fn, self.cv, self.prefac, self.omega).reshape(self.shape)
            E = self.explicit(fn) + self.boltz(fn) - P
            new = dict(F=fn.copy(), U=U, P=P, LM=self._mom(P), L=E,
                       LU=self._mom(E))
            self.hist = hs[1:] + [new]
            self.step_no += 1
            return fn
        raise ValueError(k)
