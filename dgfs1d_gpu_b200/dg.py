"""Host handle of the native nodal-DG right-hand side and stage updates."""
import ctypes

import numpy as np
import torch

from . import _native as nat
from .collision import _DT, _stream_ptr

BC_KIND = {'dgfs-periodic': 0, 'dgfs-cyclic': 0, 'dgfs-wall-diffuse': 1,
           'dgfs-inlet': 2, 'dgfs-inlet-nondim': 2, 'dgfs-vanish': 3,
           'dgfs-wall-expr-diffuse': 4}


def _dp(a):
    return ctypes.cast(a.ctypes.data, ctypes.POINTER(ctypes.c_double))


class DGOperator:
    """Advection/flux part of the DG right-hand side on (K, Ne, N^3) arrays.

    bcs: two (kind, f0, ux) triples for the left and right boundaries.
    """

    def __init__(self, basis, invjac, c0, cw, bcs):
        K, Ne, N = basis.K, len(invjac), len(c0)
        self.K, self.Ne, self.N, self.Nv = K, Ne, N, N ** 3
        self.Nqr = basis.interpMat.shape[1]
        fo = basis.faceOp
        arrs = dict(trL=fo[0], trR=fo[-1], D=basis.derivOp, gLD=basis.gLD,
                    gRD=basis.gRD, invjac=np.ravel(invjac), c0=c0,
                    im=basis.interpMat)
        self._keep = {k: np.ascontiguousarray(v, dtype=np.float64)
                      for k, v in arrs.items()}
        d = nat.DgDesc()
        d.K, d.Ne, d.N, d.Nqr = K, Ne, N, self.Nqr
        for k, v in self._keep.items():
            setattr(d, k, _dp(v))
        d.cw = float(cw)
        for s, (kind, f0, ux) in enumerate(bcs):
            d.bc_kind[s] = BC_KIND[kind]
            if f0 is not None:
                f = np.ascontiguousarray(f0, dtype=np.float64)
                self._keep['f0%d' % s] = f
                d.bc_f0[s] = _dp(f)
            d.bc_ux[s] = float(ux)
        h = ctypes.c_void_p()
        nat.check(nat.lib().dgfs_dg_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h
        if not np.array_equal(basis.invMassOp, np.eye(K)):
            raise NotImplementedError('non-identity inverse mass operator')

    def set_limiter(self, basis, invjac, xsol):
        """Tables of the linear slope limiter (abstd.py:403-415): row 0 of the
        basis' cell-average and differentiated linear-projection operators,
        the node offsets from each element centre and the element lengths,
        formed as limiters.mako forms them (h = 2/invjac, x0 = x_0 + h/2)."""
        inv = np.ravel(invjac).astype(np.float64)
        hs = (1. / inv) * 2
        xs = np.asarray(xsol, dtype=np.float64)
        dx = np.ascontiguousarray(xs - (xs[0:1, :] + hs[None, :] / 2))
        tabs = [np.ascontiguousarray(basis.cellAvgOp[0], dtype=np.float64),
                np.ascontiguousarray(basis.drLinOp[0], dtype=np.float64),
                dx, np.ascontiguousarray(hs)]
        nat.check(nat.lib().dgfs_dg_set_limiter(self._h, *[_dp(t) for t in tabs]))

    def limit(self, u, stream=None):
        """Apply the linear slope limiter to u (K, Ne, N^3) in place."""
        nat.check(nat.lib().dgfs_dg_limit(self._h, ctypes.c_void_p(u.data_ptr()),
                                          _DT[u.dtype], _stream_ptr(stream)))

    def advect(self, u, ux, stream=None):
        nat.check(nat.lib().dgfs_dg_advect(
            self._h, ctypes.c_void_p(u.data_ptr()),
            ctypes.c_void_p(ux.data_ptr()), _DT[u.dtype], _stream_ptr(stream)))

    def set_upwind(self, dpos, dneg, swap=False):
        """Use the upwind summation-by-parts volume term: dpos where c_x > 0,
        dneg where c_x < 0 (K x K); ``swap`` makes the boundaries periodic
        (each ghost takes the trace at the other end)."""
        self._keep['upw'] = [np.ascontiguousarray(dpos, dtype=np.float64),
                             np.ascontiguousarray(dneg, dtype=np.float64)]
        a, b = self._keep['upw']
        nat.check(nat.lib().dgfs_dg_set_upwind(self._h, _dp(a), _dp(b),
                                               int(bool(swap))))

    def set_entropy_stable(self, Dr):
        """Use the entropy-stable two-point volume term with the derivative
        matrix Dr (K x K, the basis' derivMat)."""
        self._keep['es'] = np.ascontiguousarray(Dr, dtype=np.float64)
        nat.check(nat.lib().dgfs_dg_set_entropy_stable(self._h, _dp(self._keep['es'])))

    def limit_positivity(self, u, stream=None):
        """Positivity limiter (limitPos) on u (K, Ne, N^3), in place; needs
        set_limiter's tables."""
        nat.check(nat.lib().dgfs_dg_limit_positivity(
            self._h, ctypes.c_void_p(u.data_ptr()), _DT[u.dtype],
            _stream_ptr(stream)))

    def set_wall_state(self, side, ux, uy, uz, T, mass=1.0):
        """Velocity and temperature (nondimensional) of a
        ``dgfs-wall-expr-diffuse`` boundary for the following advect calls."""
        nat.check(nat.lib().dgfs_dg_set_wall_state(
            self._h, int(side), float(ux), float(uy), float(uz), float(T),
            float(mass)))

    def wall_density(self):
        out = (ctypes.c_double * 2)()
        nat.check(nat.lib().dgfs_dg_wall_density(self._h, out))
        return np.array(out[:])

    def moments(self, coeff, out=None, stream=None):
        """(Nqr, Ne, 10) FP64 nondimensional moments (device tensor)."""
        if out is None:
            out = torch.empty((self.Nqr, self.Ne, 10), dtype=torch.float64,
                              device=coeff.device)
        nat.check(nat.lib().dgfs_dg_moments(
            self._h, ctypes.c_void_p(coeff.data_ptr()), _DT[coeff.dtype],
            ctypes.c_void_p(out.data_ptr()), _stream_ptr(stream)))
        return out

    def moments_bi(self, coeffs, masses, out=None, stream=None):
        """(Nqr, Ne, nspcs, 5) FP64 nondimensional mixture moments rho, Ux,
        Uy, T, Qx of the species solutions ``coeffs`` (device tensor)."""
        ns = len(coeffs)
        if out is None:
            out = torch.empty((self.Nqr, self.Ne, ns, 5), dtype=torch.float64,
                              device=coeffs[0].device)
        ptrs = (ctypes.c_void_p * ns)(*[c.data_ptr() for c in coeffs])
        ms = (ctypes.c_double * ns)(*[float(m) for m in masses])
        nat.check(nat.lib().dgfs_dg_moments_bi(
            self._h, ptrs, ns, ms, _DT[coeffs[0].dtype],
            ctypes.c_void_p(out.data_ptr()), _stream_ptr(stream)))
        return out

    def residual(self, x, y, stream=None):
        out = (ctypes.c_double * 2)()
        nat.check(nat.lib().dgfs_dg_residual(
            self._h, ctypes.c_void_p(x.data_ptr()),
            ctypes.c_void_p(y.data_ptr()), x.numel(), _DT[x.dtype], out,
            _stream_ptr(stream)))
        return out[0], out[1]

    def close(self):
        if getattr(self, '_h', None):
            nat.release(nat.lib().dgfs_dg_destroy, self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def axnpby(x0, a0, *terms, stream=None):
    """x0 <- a0 x0 + sum a_i x_i (terms = a1, x1, a2, x2, ...), in place."""
    xs = terms[1::2]
    as_ = terms[0::2]
    n = len(xs)
    ptrs = (ctypes.c_void_p * n)(*[x.data_ptr() for x in xs])
    coef = (ctypes.c_double * n)(*[float(a) for a in as_])
    nat.check(nat.lib().dgfs_axnpby(
        ctypes.c_void_p(x0.data_ptr()), x0.numel(), _DT[x0.dtype], float(a0),
        n, ptrs, coef, _stream_ptr(stream)))
