"""Penalised IMEX time integrators (``[time-integrator] scheme``).

Keys and coefficients of dgfs1D/astd/integrator.py: ``bdf-111`` / ``bdf-222`` /
``bdf-333`` (penalty model only, explicit DG advection; :281-488), ``boltz-ars-111``
(explicit Boltzmann operator and penalty, :491-552) and ``imex-lm-bdf1`` /
``imex-lm-bdf2`` and the other ``imex-lm-*`` schemes (cn2, ad2, sg2, bdf3,
ad3, tvb3, bdf4, tvb4, shu3, shu4; explicit L + Q - P, implicit P(f^{n+1});
:623-907).  The
moment update is the linear combination of the scheme followed by the
penalty model's implicit relaxation of its non-conserved moments (the
updateMoment{BDF,LM} kernels of the model).
Differences from the reference, all in start-up or dead code: the s - 1
start-up levels come from first-order substeps of the same family (the
reference uses ARS-222/443 substeps); the explicit part of a new IMEX-LM level uses
that level's penalty P(f^{n+1}) (the reference's two-stage path would use
the previous level's after its circular shift, but exits the process after
its first step, astd/integrator.py:732, so it never gets there).
"""
import torch

from ..dg import axnpby


def _lin(out, pairs):
    """out = sum a_i x_i over (a, x) pairs, in chunks of the native axnpby."""
    pairs = [(a, x) for a, x in pairs if a != 0.0]
    if not pairs:
        out.zero_()
        return
    first = True
    while pairs:
        chunk, pairs = pairs[:4 if first else 3], pairs[4 if first else 3:]
        terms = []
        for a, x in chunk:
            terms += [a, x]
        axnpby(out, 0.0 if first else 1.0, *terms)
        first = False


class DGFSIntegratorAstd:
    intg_kind = None

    def __init__(self, explicit, sm, shape, dtype, t=0.0, dt=None, f0=None,
                 explicitQ=None, nsub=10, device='cuda', **kwargs):
        self._explicit, self._sm, self._Q = explicit, sm, explicitQ
        self.shape, self.dtype, self.device = shape, dtype, device
        self.npts = shape[0] * shape[1]
        self.dt, self.nsub = dt, nsub

    def _z(self):
        return torch.zeros(self.shape, dtype=self.dtype, device=self.device)

    def _zm(self):
        return torch.zeros((self.npts, self._sm.nalph), dtype=torch.float64,
                           device=self.device)

    def _mom(self, x):
        U = self._zm()
        self._sm.moment(0.0, x, U)
        return U


class Bdf111IntegratorAstd(DGFSIntegratorAstd):
    intg_kind = 'bdf-111'

    def integrate(self, t, dt, nacptsteps, f):
        U0 = self._mom(f)
        L0 = self._z()
        self._explicit(t, f, L0)
        LU0 = self._mom(L0)
        U = self._zm()
        _lin(U, [(1.0, U0), (dt, LU0)])
        self._sm.relax(U, 1.0, dt)
        rhs = self._z()
        _lin(rhs, [(1.0, f), (dt, L0)])
        self._sm.implicit(U, rhs, f, 1.0, dt)


class _StageIMEXIntegratorAstd(DGFSIntegratorAstd):
    """Penalty-only IMEX Runge-Kutta schemes of the linear kinetic driver
    (dgfsAstd1D) with the BGK model: ARS (astd/integrator.py:56-179) and SSPL
    (:182-278) with the updateMom{q}_ARS / updateDistribution{q}_ARS /
    updateDistributionWeight{q}_SSPL arithmetic of bgk-direct-gll.mako:202-326.
    With stage moments U_j, stage solutions F_j, L_j the advection of a stage
    and P_j = nu(U_j) (M(U_j) - F_j):
      U_q = U_0 + dt sum_j _a_qj LU_j
      F_q = (F_0 + dt sum_j _a_qj L_j + dt sum_{j<q} a_qj P_j
             + a_qq dt nu_q M_q) / (1 + a_qq dt nu_q).
    Not built with a Boltzmann operator (in the Boltzmann drivers the
    reference's ARS stage overwrites Q(f) before using it) nor for the
    ES-BGK / Shakov models."""

    def __init__(self, explicit, sm, shape, dtype, explicitQ=None, **kwargs):
        super().__init__(explicit, sm, shape, dtype, explicitQ=explicitQ, **kwargs)
        if explicitQ is not None:
            raise NotImplementedError('%s with a Boltzmann operator' % self.intg_kind)
        if sm.kind != 0:
            raise NotImplementedError('%s with the %s model' % (
                self.intg_kind, sm.scattering_model))

    def _stage(self, t, dt, F0, Ls, Ps, q_expl, q_impl, U):
        """F_q from the explicit weights over Ls, implicit weights over the
        earlier stages' penalties Ps and the implicit weight of stage q."""
        rhs = self._z()
        _lin(rhs, [(1.0, F0)] + [(dt * a, L) for a, L in zip(q_expl, Ls)]
             + [(dt * a, P) for a, P in zip(q_impl, Ps)])
        f = self._z()
        self._sm.implicit(U, rhs, f, 1.0, self._aqq * dt)
        return f

    def _penalty(self, t, U, f):
        P = self._z()
        self._sm.collide(t, U, f, P)
        return P


class ARSIntegratorAstd(_StageIMEXIntegratorAstd):
    intg_kind = None
    _A = A = None

    def integrate(self, t, dt, nacptsteps, f):
        ns = len(self.A) - 1
        F0 = f.clone()
        U0 = self._mom(F0)
        Fs, Us, Ls, LUs, Ps = [F0], [U0], [], [], []
        for i in range(ns):
            L = self._z()
            self._explicit(t, Fs[i], L)
            Ls.append(L)
            LUs.append(self._mom(L))
            ex = self._A[i + 1][0:i + 1]
            U = self._zm()
            _lin(U, [(1.0, U0)] + [(dt * a, LU) for a, LU in zip(ex, LUs)])
            Us.append(U)
            self._aqq = self.A[i + 1][i + 1]
            Fq = self._stage(t, dt, F0, Ls, Ps, ex, self.A[i + 1][1:i + 1], U)
            Fs.append(Fq)
            if i + 1 < ns:
                Ps.append(self._penalty(t, U, Fq))
        f.copy_(Fs[-1])


class ARS111IntegratorAstd(ARSIntegratorAstd):
    intg_kind = 'ars-111'
    _A = [[0., 0.], [1., 0.]]
    A = [[0., 0.], [0., 1.]]


class ARS222IntegratorAstd(ARSIntegratorAstd):
    intg_kind = 'ars-222'
    _g = 1. - (2. ** 0.5) / 2.
    _d = 1. - 1. / (2. * _g)
    _A = [[0., 0., 0.], [_g, 0., 0.], [_d, 1 - _d, 0.]]
    A = [[0., 0., 0.], [0., _g, 0.], [0., 1 - _g, _g]]


class ARS443IntegratorAstd(ARSIntegratorAstd):
    intg_kind = 'ars-443'
    _A = [[0., 0., 0., 0., 0.], [1. / 2., 0., 0., 0., 0.],
          [11. / 18., 1. / 18., 0., 0., 0.], [5. / 6., -5. / 6., 1. / 2., 0., 0.],
          [1. / 4., 7. / 4., 3. / 4., -7. / 4., 0.]]
    A = [[0., 0., 0., 0., 0.], [0., 1. / 2., 0., 0., 0.], [0., 1. / 6., 1. / 2., 0., 0.],
         [0., -1. / 2., 1. / 2., 1. / 2., 0.], [0., 3. / 2., -3. / 2., 1. / 2., 1. / 2.]]


class SSPLIntegratorAstd(_StageIMEXIntegratorAstd):
    """SSP L-stable schemes: the first stage is implicit only, stage q uses
    row q-1 of the tables (a_qj = A[q-1][j-1]), and the new solution is the
    weighted sum F_0 + dt sum_j (_w_j L_j + w_j P_j) over all stages."""
    intg_kind = None
    _A = A = _w = w = None

    def integrate(self, t, dt, nacptsteps, f):
        ns = len(self.A)
        F0 = f.clone()
        U0 = self._mom(F0)
        U1 = U0.clone()
        self._aqq = self.A[0][0]
        F1 = self._stage(t, dt, F0, [], [], [], [], U1)
        Fs, Us, Ls, LUs, Ps = [F0, F1], [U0, U1], [], [], [self._penalty(t, U1, F1)]
        for i in range(1, ns):
            L = self._z()
            self._explicit(t, Fs[i], L)
            Ls.append(L)
            LUs.append(self._mom(L))
            ex = self._A[i][0:i]
            U = self._zm()
            _lin(U, [(1.0, U0)] + [(dt * a, LU) for a, LU in zip(ex, LUs)])
            Us.append(U)
            self._aqq = self.A[i][i]
            Fq = self._stage(t, dt, F0, Ls, Ps, ex, self.A[i][0:i], U)
            Fs.append(Fq)
            Ps.append(self._penalty(t, U, Fq))
        L = self._z()
        self._explicit(t, Fs[ns], L)
        Ls.append(L)
        _lin(f, [(1.0, F0)] + [(dt * a, x) for a, x in zip(self._w, Ls)]
             + [(dt * a, P) for a, P in zip(self.w, Ps)])


class SSPL222IntegratorAstd(SSPLIntegratorAstd):
    intg_kind = 'sspl-222'
    _g = 1. - (2. ** 0.5) / 2.
    _A = [[0., 0.], [1., 0.]]
    A = [[_g, 0.], [1 - 2 * _g, _g]]
    _w = [0.5, 0.5]
    w = [0.5, 0.5]


class SSPL443IntegratorAstd(SSPLIntegratorAstd):
    intg_kind = 'sspl-443'
    _al, _be, _et = 0.24169426078821, 0.06042356519705, 0.12915286960590
    _A = [[0., 0., 0., 0.], [0., 0., 0., 0.], [0., 1., 0., 0.], [0., 1. / 4., 1. / 4., 0.]]
    A = [[_al, 0., 0., 0.], [-_al, _al, 0., 0.], [0., 1. - _al, _al, 0.],
         [_be, _et, 1. / 2. - _be - _et - _al, _al]]
    _w = [0., 1. / 6., 1. / 6., 2. / 3.]
    w = [0., 1. / 6., 1. / 6., 2. / 3.]


class BoltzARS111IntegratorAstd(DGFSIntegratorAstd):
    """First-order ARS scheme of the penalised Boltzmann equation
    (astd/integrator.py:491-552): the moments advance with the advection
    only; f advances with the explicit L + Q(f) - P(f), P = nu (M(U^n) - f),
    and the implicit penalty at the new moments."""
    intg_kind = 'boltz-ars-111'

    def integrate(self, t, dt, nacptsteps, f):
        U0 = self._mom(f)
        P0 = self._z()
        self._sm.collide(t, U0, f, P0)
        L0 = self._z()
        self._explicit(t, f, L0)
        LU0 = self._mom(L0)
        if self._Q is not None:
            self._Q(t, f, L0)             # accumulates Q(f)
        axnpby(L0, 1.0, -1.0, P0)
        U = self._zm()
        _lin(U, [(1.0, U0), (dt, LU0)])
        self._sm.relax(U, 1.0, dt)
        rhs = self._z()
        _lin(rhs, [(1.0, f), (dt, L0)])
        self._sm.implicit(U, rhs, f, 1.0, dt)


class BdfIntegratorAstd(DGFSIntegratorAstd):
    """k-level BDF penalty schemes (astd/integrator.py:325-488): with levels
    n-k+1 .. n, U = sum_i (-A_i U_i + G_i dt LU_i) / A_k relaxed with
    (A_k, B dt), then f = (sum_i (-A_i f_i + G_i dt L_i) + B dt nu M(U)) /
    (A_k + B dt nu).  Levels 1 .. k-1 come from nsub first-order substeps
    each, one level per step (the reference uses ARS-222 substeps and, for
    bdf-333, computes two levels in its first step)."""
    intg_kind = None
    A = G = B = None

    def _state(self, t, f):
        L = self._z()
        self._explicit(t, f, L)
        return dict(F=f.clone(), U=self._mom(f), L=L, LU=self._mom(L))

    def integrate(self, t, dt, nacptsteps, f):
        A, G, B = self.A, self.G, self.B
        k = len(G)
        if nacptsteps < k - 1:
            if nacptsteps == 0:
                self.hist = [self._state(t, f)]
            sub = Bdf111IntegratorAstd(self._explicit, self._sm, self.shape,
                                       self.dtype, device=self.device)
            for i in range(self.nsub):
                sub.integrate(t + i * dt / self.nsub, dt / self.nsub, i, f)
            self.hist.append(self._state(t + dt, f))
            return
        hs = self.hist
        U = self._zm()
        _lin(U, [p for i in range(k) for p in (
            (-A[i] / A[k], hs[i]['U']), (G[i] * dt / A[k], hs[i]['LU']))])
        self._sm.relax(U, A[k], B * dt)
        rhs = self._z()
        _lin(rhs, [p for i in range(k) for p in (
            (-A[i], hs[i]['F']), (G[i] * dt, hs[i]['L']))])
        self._sm.implicit(U, rhs, f, A[k], B * dt)
        self.hist = hs[1:] + [self._state(t + dt, f)]


class Bdf222IntegratorAstd(BdfIntegratorAstd):
    intg_kind = 'bdf-222'
    A = [1. / 3., -4. / 3., 1.]
    G = [-2. / 3., 4. / 3.]
    B = 2. / 3.


class Bdf333IntegratorAstd(BdfIntegratorAstd):
    intg_kind = 'bdf-333'
    A = [-2. / 11., 9. / 11., -18. / 11., 1.]
    G = [6. / 11., -18. / 11., 18. / 11.]
    B = 6. / 11.


class IMEXLMIntegratorAstd(DGFSIntegratorAstd):
    intg_kind = None
    A = B = C = None

    def __init__(self, explicit, sm, shape, dtype, t=0.0, dt=None, f0=None,
                 explicitQ=None, **kwargs):
        super().__init__(explicit, sm, shape, dtype, t=t, dt=dt, f0=f0,
                         explicitQ=explicitQ, **kwargs)
        s = len(self.A)
        self.hist = [self._state(t, f0)]
        self.starts = []
        if s > 1:
            # levels 1 .. s-1 by nsub first-order substeps each, continuing
            f = f0.clone()
            sub = IMEXLMBdf1IntegratorAstd(explicit, sm, shape, dtype, t=t,
                                           dt=dt / self.nsub, f0=f,
                                           explicitQ=explicitQ,
                                           device=self.device)
            k = 0
            for lvl in range(1, s):
                for _ in range(self.nsub):
                    sub.integrate(t + k * dt / self.nsub, dt / self.nsub, k, f)
                    k += 1
                self.starts.append(f.clone())
                self.hist.append(self._state(t + lvl * dt, f))

    def _state(self, t, f):
        U = self._mom(f)
        P = self._z()
        self._sm.collide(t, U, f, P)
        E = self._z()
        self._explicit(t, f, E)
        if self._Q is not None:
            self._Q(t, f, E)          # accumulates Q(f)
        axnpby(E, 1.0, -1.0, P)
        return dict(F=f.clone(), U=U, P=P, LM=self._mom(P), L=E,
                    LU=self._mom(E))

    def integrate(self, t, dt, nacptsteps, f):
        A, B, C = self.A, self.B, self.C
        s = len(A)
        if nacptsteps < s - 1:
            f.copy_(self.starts[nacptsteps])
            return
        hs = self.hist
        U = self._zm()
        _lin(U, [p for i in range(s) for p in (
            (-A[s - i - 1], hs[i]['U']), (dt * B[s - i - 1], hs[i]['LU']),
            (dt * C[s - i], hs[i]['LM']))])
        rhs = self._z()
        _lin(rhs, [p for i in range(s) for p in (
            (-A[s - i - 1], hs[i]['F']), (dt * B[s - i - 1], hs[i]['L']),
            (dt * C[s - i], hs[i]['P']))])
        self._sm.relax(U, 1.0, C[0] * dt)
        P = self._z()
        self._sm.implicit(U, rhs, f, 1.0, C[0] * dt, P=P)
        E = self._z()
        self._explicit(t + dt, f, E)
        if self._Q is not None:
            self._Q(t + dt, f, E)
        axnpby(E, 1.0, -1.0, P)
        new = dict(F=f.clone(), U=U, P=P, LM=self._mom(P), L=E,
                   LU=self._mom(E))
        self.hist = hs[1:] + [new]


class IMEXLMBdf1IntegratorAstd(IMEXLMIntegratorAstd):
    intg_kind = 'imex-lm-bdf1'
    A, B, C = [-1.], [1.], [1., 0.]


class IMEXLMBdf2IntegratorAstd(IMEXLMIntegratorAstd):
    intg_kind = 'imex-lm-bdf2'
    A, B, C = [-4. / 3., 1. / 3.], [4. / 3., -2. / 3.], [2. / 3., 0., 0.]


# The remaining IMEX linear multistep schemes of astd/integrator.py:751-907
# (coefficient tables kept as the reference defines them: A, B of length s,
# C of length s + 1).
_LM_SCHEMES = {
    'imex-lm-cn2': ([-1., 0.], [1.5, -0.5], [0.5, 0.5, 0.]),
    'imex-lm-ad2': ([-1., 0.], [1.5, -0.5], [9. / 16., 3. / 8., 1. / 16.]),
    'imex-lm-sg2': ([-3. / 4., 0., -1. / 4.], [3. / 2., 0., 0.],
                    [1., 0., 0., 1. / 2.]),
    'imex-lm-bdf3': ([-18. / 11., 9. / 11., -2. / 11.],
                     [18. / 11., -18. / 11., 6. / 11.], [6. / 11., 0., 0., 0.]),
    'imex-lm-ad3': ([-1., 0., 0.], [23. / 12., -4. / 3., 5. / 12.],
                    [4661. / 10000., 15551. / 30000., 1949. / 30000.,
                     -1483. / 30000.]),
    'imex-lm-tvb3': ([-3909. / 2048., 1367. / 1024., -873. / 2048.],
                     [18463. / 12288., -1271. / 768., 8233. / 12288.],
                     [1089. / 2048., -1139. / 12288., -367. / 6144.,
                      1699. / 12288.]),
    'imex-lm-bdf4': ([-48. / 25., 36. / 25., -16. / 25., 3. / 25.],
                     [48. / 25., -72. / 25., 48. / 25., -12. / 25.],
                     [12. / 25., 0., 0., 0., 0.]),
    'imex-lm-tvb4': ([-21531. / 8192., 22753. / 8192., -12245. / 8192.,
                      2831. / 8192.],
                     [13261. / 8192., -75029. / 24576., 54799. / 24576.,
                      -15245. / 24576.],
                     [4207. / 8192., -3567. / 8192., 697. / 24576.,
                      4315. / 24576., -41. / 384.]),
    'imex-lm-shu3': ([-16. / 27, 0., 0., -11. / 27.], [16. / 9., 0., 0., 4. / 9.],
                     [9035. / 19683., 13541. / 19683., 1127. / 2187.,
                      7927. / 19683., 3094. / 19683.]),
    'imex-lm-shu4': ([-137. / 400., 0., 0., -959. / 5000., -8781. / 94000.,
                      -87487 / 235000.],
                     [976903. / 470000., 0., 0., 136757. / 117500.,
                      266997. / 470000., 0.],
                     [237. / 500., 7547. / 10000., 299. / 400., 4513. / 5875.,
                      118099. / 235000., 174527. / 470000., 90349. / 470000.]),
}
for _kind, (_A, _B, _C) in _LM_SCHEMES.items():
    globals()['IMEXLM_%s_IntegratorAstd' % _kind.split('-')[-1].upper()] = type(
        'IMEXLM_%s_IntegratorAstd' % _kind.split('-')[-1].upper(),
        (IMEXLMIntegratorAstd,), dict(intg_kind=_kind, A=_A, B=_B, C=_C))
