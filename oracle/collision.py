"""Oracle restatement of the fast-spectral collision operators (float64).

Test infrastructure only (see ``oracle/__init__.py``).  Each function follows
the reference kernel sequence literally -- one FFT per (p, q) term, no
linearity or symmetry savings -- so that it is a faithful checker of the
restructured GPU kernels.

cuFFT conventions: ``_fwd(x) = fftn(x)`` (CUFFT_FORWARD, unnormalised) and
``_inv(x) = n * ifftn(x)`` (CUFFT_INVERSE, unnormalised).
"""
import os

import numpy as np
import scipy.fft as sfft

from .mesh import fft_lvectors

_WORKERS = int(os.environ.get('DGFS_ORACLE_WORKERS', os.cpu_count() or 1))


def _fwd(x, axes=(-3, -2, -1)):
    return sfft.fftn(x, axes=axes, workers=_WORKERS)


def _inv(x, axes=(-3, -2, -1)):
    return sfft.ifftn(x, axes=axes, norm='forward', workers=_WORKERS)


def sinc(s, eps=1e-15):
    """sin(s+eps)/(s+eps) (vhs-gll.mako:9-23; eps=1e-6 in float mode)."""
    return np.sin(s + eps) / (s + eps)


class VHSTables:
    """a, b1, b2 tables of the VHS model.

    Restates ``precompute_aa`` / ``precompute_bb`` (vhs-gll.mako:43-99) and
    the l-vectors of std/scattering.py:116-128.  ``sphere_factor`` is the 2 of
    computeQG (vhs-gll.mako:192) for the half-sphere rule, 1 for a full one.
    """

    def __init__(self, N, L, qz, qw, sz, sw, gamma, sphere_factor=2.0,
                 eps=1e-15):
        self.N, self.n = N, N ** 3
        self.L, self.qz, self.qw = L, np.asarray(qz), np.asarray(qw)
        self.sz, self.sw, self.gamma = np.asarray(sz), sw, gamma
        self.sphere_factor = sphere_factor
        lx, ly, lz = fft_lvectors(N)
        Nrho, M = len(qz), len(sz)
        self.aa = np.empty((Nrho, M, self.n))
        for p in range(Nrho):
            fac = np.pi / L * qz[p] / 2.
            for q in range(M):
                self.aa[p, q] = fac * ((sz[q, 0] * lx) + (sz[q, 1] * ly)
                                       + (sz[q, 2] * lz))
        cSqr = np.sqrt(lx * lx + ly * ly + lz * lz)
        self.bb1 = np.empty((Nrho, self.n))
        self.bb2 = np.zeros(self.n)
        for p in range(Nrho):
            self.bb1[p] = (pow(qz[p], gamma + 2.) * 4 * np.pi
                           * sinc(np.pi / L * qz[p] / 2. * cSqr, eps))
            self.bb2 += (qw[p] * pow(qz[p], gamma + 2.) * 16 * np.pi * np.pi
                         * sinc(np.pi / L * qz[p] * cSqr, eps))


def vhs_gll_fs(tab, prefac, f):
    """One ``DGFSVHSGLLScatteringModelStd.fs`` evaluation: returns Q(f, f).

    Restates std/scattering.py:251-313 with the kernels r2z_, cosSinMul,
    magSqr, computeQG, ax and output_append_ (vhs-gll.mako:101-218, 399-433).
    The reference *accumulates* prefac*(...) into Q; this returns the
    increment.
    """
    N, n = tab.N, tab.n
    Nrho, M = tab.aa.shape[:2]
    fC = f.reshape(N, N, N).astype(np.complex128)
    FTf = _fwd(fC) / n
    a = tab.aa.reshape(Nrho, M, N, N, N)
    intw = tab.sphere_factor * tab.qw * tab.sw / n
    bb1 = tab.bb1.reshape(Nrho, N, N, N)
    # the reference's batched plans run all Nrho*M terms at once; here one
    # radial point at a time (same terms, bounded memory at N=48)
    QGh = np.zeros((N, N, N), dtype=np.complex128)
    for p in range(Nrho):
        t1 = np.cos(a[p]) * FTf
        t2 = np.sin(a[p]) * FTf
        t3 = _inv(t1)
        t4 = _inv(t2)
        t2 = t3 * t3 + t4 * t4
        t1 = _fwd(t2)
        QGh += intw[p] * bb1[p] * t1.sum(axis=0)
    QG = _inv(QGh)
    fL = _inv(tab.bb2.reshape(N, N, N) * FTf)
    return (prefac * (QG.real - f.reshape(N, N, N) * fL.real)).ravel()


def vhs_fs(tab, prefac, f, g):
    """Bilinear ``DGFSVHSScatteringModelStd.fs`` (std/scattering.py:346-429).

    Gain from IFFT(cos a F) IFFT(cos a G) + IFFT(sin a F) IFFT(sin a G)
    (cosMul/sinMul/cplxMul/cplxMulAdd, vhs-gll.mako:260-397); loss
    f * IFFT(b2 G).
    """
    N, n = tab.N, tab.n
    Nrho, M = tab.aa.shape[:2]
    FTf = _fwd(f.reshape(N, N, N).astype(np.complex128)) / n
    FTg = _fwd(g.reshape(N, N, N).astype(np.complex128)) / n
    a = tab.aa.reshape(Nrho, M, N, N, N)
    ca, sa = np.cos(a), np.sin(a)
    t5 = _inv(ca * FTf) * _inv(ca * FTg)
    t5 = t5 + _inv(sa * FTf) * _inv(sa * FTg)
    t1 = _fwd(t5)
    intw = (tab.sphere_factor * tab.qw * tab.sw / n)[:, None, None, None]
    QGh = np.sum(intw * tab.bb1.reshape(Nrho, N, N, N) * t1.sum(axis=1),
                 axis=0)
    QG = _inv(QGh)
    fL = _inv(tab.bb2.reshape(N, N, N) * FTg)
    return (prefac * (QG.real - f.reshape(N, N, N) * fL.real)).ravel()


class VSSTables:
    """a, b_pq and c_pq tables of the VSS mixture model for one pair (p, q).

    Restates ``precompute_a`` and ``precompute_bc_pq`` (vss.mako:29-93) with
    the launch loop of bi/scattering.py:185-204.  ``szpre`` is the Mpre-point
    full-sphere rule, ``eta`` = alpha-1, ``mpq`` = m_q/(m_p+m_q).
    """

    def __init__(self, N, L, qz, qw, sz, sw, szpre, gamma, eta, mpq):
        self.N, self.n = N, N ** 3
        lx, ly, lz = fft_lvectors(N)
        Nrho, M = len(qz), len(sz)
        Mpre = len(szpre)
        swpre = 4 * np.pi / Mpre
        self.aa = np.empty((Nrho, M, self.n))
        self.b = np.empty((Nrho, M, self.n), dtype=np.complex128)
        self.c = np.zeros(self.n, dtype=np.complex128)
        self.qw, self.sw = np.asarray(qw), sw
        szpre = np.asarray(szpre)
        # Bpq[y, k] = (1 + sigma_y . sigma'_k)^eta, the kernel weight of the
        # precompute loop (one launch per (x, y), a sum over k inside)
        Bpq = np.power(1 + np.asarray(sz) @ szpre.T, eta)
        lmat = np.stack([lx, ly, lz])
        for x in range(Nrho):
            fac = np.pi / L * qz[x]
            fac_b = swpre * pow(qz[x], gamma + 2)
            fac_c = qw[x] * sw * fac_b
            Ld = fac * (szpre @ lmat)                       # [Mpre, n]
            # sum_k Bpq[y,k] fac_b e^{-i mpq Ld_k}, sum_k Bpq[y,k] fac_c e^{-i Ld_k}
            self.b[x] = fac_b * (Bpq @ np.exp(-1j * mpq * Ld))
            self.c += fac_c * np.sum(Bpq @ np.exp(-1j * Ld), axis=0)
            for y in range(M):
                self.aa[x, y] = fac * (sz[y, 0] * lx + sz[y, 1] * ly
                                       + sz[y, 2] * lz)


def vss_fs(tab, prefac, mp, mq, f1, f2):
    """One ``DGFSBiVSSScatteringModel.fs`` pair evaluation: Q_pq(f_p, f_q).

    Restates bi/scattering.py:263-321 with r2z, cosSinMul_pq, prod,
    computeQG, ax2 and output_pq (vss.mako:96-286).
    """
    N, n = tab.N, tab.n
    Nrho, M = tab.aa.shape[:2]
    FTf = _fwd(f1.reshape(N, N, N).astype(np.complex128)) / n
    FTg = _fwd(f2.reshape(N, N, N).astype(np.complex128)) / n
    a = tab.aa.reshape(Nrho, M, N, N, N)
    t1 = np.exp(1j * a * (mq / (mp + mq))) * FTf
    t2 = np.exp(-1j * a * (mp / (mp + mq))) * FTg
    t3 = _inv(t1)
    t1 = _inv(t2)
    t2 = t3 * t1
    t1 = _fwd(t2)
    intw = (tab.qw * tab.sw / n)[:, None, None, None, None]
    QGh = np.sum(intw * tab.b.reshape(Nrho, M, N, N, N) * t1, axis=(0, 1))
    QG = _inv(QGh)
    fL = _inv(tab.c.reshape(N, N, N) * FTg)
    return (prefac * (QG.real - f1.reshape(N, N, N) * fL.real)).ravel()
