"""Oracle restatement of the host-side setup: quadratures, velocity meshes,
spherical designs and collision-kernel prefactors (float64, NumPy).

Test infrastructure only (see ``oracle/__init__.py``).
"""
import math
import os

import numpy as np

_DESIGNS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(
    __file__))), 'dgfs1d_gpu_b200', 'data', 'womersley_symmetric.npz')


# -- quadratures -------------------------------------------------------------

def jacobi_recurrence(n, a, b):
    """Monic Jacobi three-term recurrence (alpha_k, beta_k).

    Restates ``rjacobi`` (dgfs1D/quadratures.py:171-193).
    """
    ra, rb = np.zeros(n), np.zeros(n)
    apbp2 = 2. + a + b
    ra[0] = (b - a) / apbp2
    rb[0] = 2.0 ** (a + b + 1) * (math.gamma(a + 1.) * math.gamma(b + 1.)
                                  / math.gamma(apbp2))
    if n > 1:
        rb[1] = 4. * (a + 1.) * (b + 1.) / ((apbp2 + 1.) * apbp2 * apbp2)
    apbp2 += 2
    for i in range(1, n - 1):
        ra[i] = (b * b - a * a) / ((apbp2 - 2.) * apbp2)
        rb[i + 1] = (4. * (i + 1) * (i + 1 + a) * (i + 1 + b) * (i + 1 + a + b)
                     / ((apbp2 * apbp2 - 1) * apbp2 * apbp2))
        apbp2 += 2
    ra[n - 1] = (b * b - a * a) / ((apbp2 - 2.) * apbp2)
    return ra, rb


def golub_welsch(ra, rb):
    """Nodes/weights from the symmetric tridiagonal Jacobi matrix.

    Restates ``gauss`` (dgfs1D/quadratures.py:195-204).
    """
    rb = rb.copy()
    scal = rb[0]
    rb[:-1] = np.sqrt(rb[1:])
    z, V = np.linalg.eigh(np.diag(ra) + np.diag(rb[:-1], -1))
    idx = np.argsort(z)
    z = z[idx]
    w = scal * V[0, idx] ** 2
    return z, w


def gauss_jacobi(n, a=0., b=0.):
    """Gauss-Jacobi rule on [-1, 1] (``zwgj``, dgfs1D/quadratures.py:205-208)."""
    return golub_welsch(*jacobi_recurrence(n, a, b))


def gauss_lobatto_jacobi(n, a=0., b=0.):
    """Gauss-Lobatto-Jacobi rule (``zwglj``, dgfs1D/quadratures.py:209-220)."""
    N = n - 2
    z, w = jacobi_recurrence(n, a, b)
    apb1 = a + b + 1.
    z[n - 1] = (a - b) / (2. * N + apb1 + 1.)
    w[n - 1] = (4. * (N + a + 1.) * (N + b + 1.) * (N + apb1)
                / ((2. * N + apb1) * (2 * N + apb1 + 1) ** 2.))
    return golub_welsch(z, w)


def jacobi_poly(n, a, b, z):
    """P_0..P_n via the three-term recurrence (dgfs1D/quadratures.py:8-28)."""
    j = [np.ones_like(z)]
    if n >= 1:
        j.append(((a + b + 2) * z + a - b) / 2)
    if n >= 2:
        apb, bbmaa = a + b, b * b - a * a
        for q in range(2, n + 1):
            qapbpq, apbp2q = q * (apb + q), apb + 2 * q
            apbp2qm1, apbp2qm2 = apbp2q - 1, apbp2q - 2
            aq = apbp2q * apbp2qm1 / (2 * qapbpq)
            bq = apbp2qm1 * bbmaa / (2 * qapbpq * apbp2qm2)
            cq = apbp2q * (a + q - 1) * (b + q - 1) / (qapbpq * apbp2qm2)
            j.append((aq * z - bq) * j[-1] - cq * j[-2])
    return j


def jacobi_poly_diff(n, a, b, z):
    """Derivatives of P_0..P_n (dgfs1D/quadratures.py:30-37)."""
    dj = [np.zeros_like(z)]
    if n >= 1:
        dj.extend(jp * (i + a + b + 2) / 2
                  for i, jp in enumerate(jacobi_poly(n - 1, a + 1, b + 1, z)))
    return dj


def ortho_basis_at(order, pts):
    """Orthonormal Legendre basis, shape (order, npts) (quadratures.py:39-51)."""
    pts = np.asarray(pts, dtype=np.float64)
    jp = jacobi_poly(order - 1, 0, 0, pts)
    return np.array([np.sqrt(i + 0.5) * p for i, p in enumerate(jp)])


def jac_ortho_basis_at(order, pts):
    """d/dz of the orthonormal basis, shape (order, npts)."""
    pts = np.asarray(pts, dtype=np.float64)
    djp = jacobi_poly_diff(order - 1, 0, 0, pts)
    return np.array([np.sqrt(i + 0.5) * p for i, p in enumerate(djp)])


def nodal_basis_at(order, pts, epts):
    """Lagrange basis on ``pts`` evaluated at ``epts`` (quadratures.py:59-61)."""
    return np.linalg.solve(ortho_basis_at(order, pts),
                           ortho_basis_at(order, epts)).T


def jac_nodal_basis_at(order, pts, epts):
    """Derivative of the Lagrange basis (quadratures.py:63-65)."""
    return np.linalg.solve(ortho_basis_at(order, pts),
                           jac_ortho_basis_at(order, epts))


# -- spherical designs -------------------------------------------------------

def sphere_design(npts, path=_DESIGNS):
    """Womersley symmetric design with ``npts`` points (highest degree).

    Restates the file selection of dgfs1D/sphericaldesign/__init__.py:62-80.
    """
    data = np.load(path)
    best = None
    for key in data.files:
        deg, m = int(key[2:5]), int(key[7:])
        if m == npts and (best is None or deg > best[0]):
            best = (deg, key)
    if best is None:
        raise ValueError('No suitable spherical quadrature rule found')
    return np.array(data[best[1]])


# -- velocity meshes ---------------------------------------------------------

R0 = 8.3144598
NA = 6.0221409e+23


class VelocityMeshStd:
    """Single-species velocity mesh (dgfs1D/std/velocitymesh.py:24-105).

    Parameters are the INI values: H0, T0, rho0, molarMass0, Nv, Nrho, cmax,
    Tmax, dev, M (half-sphere count: the 2M-point design's first M points).
    ``full_sphere=True`` instead loads the M-point design with weight 4pi/M
    (the mixture convention, bi/velocitymesh.py:111-119).
    """

    def __init__(self, Nv, M, Nrho=None, dev=5., cmax=0., Tmax=273., T0=273.,
                 H0=1e-3, rho0=1e-4, molarMass0=39.96e-3, full_sphere=False):
        self.H0, self.T0, self.rho0, self.molarMass0 = H0, T0, rho0, molarMass0
        self.n0 = rho0 / molarMass0 * NA
        self.u0 = math.sqrt(2 * R0 / molarMass0 * T0)
        self.Nv = Nv
        self.vsize = Nv ** 3
        self.Nrho = int(Nv / 2) if Nrho is None else Nrho
        cmax = cmax / self.u0
        Tmax = Tmax / T0
        self.L = cmax + dev * np.sqrt(Tmax)
        self.S = self.L * 2.0 / (3.0 + np.sqrt(2.0))
        self.R = 2 * self.S
        self.cw = (2.0 * self.L / Nv) ** 3
        c0 = np.linspace(-self.L + self.L / Nv, self.L - self.L / Nv, Nv)
        g = np.meshgrid(c0, c0, c0, indexing='ij')
        self.cv = np.stack([x.ravel() for x in g])
        qz, qw = gauss_jacobi(self.Nrho, 0., 0.)
        self.qz = (self.R / 2.0) * (1.0 + qz)
        self.qw = ((self.R - 0.0) / 2.0) * qw
        self.M = M
        if full_sphere:
            self.sz = sphere_design(M)
            self.sw = 4 * np.pi / M
            self.sphere_factor = 1.0
        else:
            self.sz = sphere_design(2 * M)[0:M, :]
            self.sw = 2 * np.pi / M
            self.sphere_factor = 2.0


class VelocityMeshBi:
    """Binary-mixture velocity mesh (dgfs1D/bi/velocitymesh.py:24-119)."""

    def __init__(self, Nv, M, masses, Nrho=None, dev=5., cmax=0., Tmax=273.,
                 T0=273., H0=1e-3, rho0=1e-4, molarMass0=39.96e-3):
        self.H0, self.T0, self.rho0, self.molarMass0 = H0, T0, rho0, molarMass0
        self.n0 = rho0 / molarMass0 * NA
        self.u0 = math.sqrt(2 * R0 / molarMass0 * T0)
        self.Nv = Nv
        self.vsize = Nv ** 3
        self.Nrho = int(Nv / 2) if Nrho is None else Nrho
        self.masses = list(masses)
        mr = max(self.masses)
        assert mr <= 4, 'Mass ratio is too high!'
        cmax = cmax / self.u0
        Tmax = Tmax / T0
        self.L = cmax + dev * np.sqrt(Tmax)
        self.S = min(
            self.L * 2.0 / (max(4. * mr / (1. + mr), 2.) + np.sqrt(1. + mr) + 1.),
            self.L * 2.0 / (max(4. * 1. / (1. + mr), 2.) + np.sqrt(1. + 1.0 / mr)
                            + 1.0))
        self.R = 2 * self.S
        self.cw = (2.0 * self.L / Nv) ** 3
        c0 = np.linspace(-self.L + self.L / Nv, self.L - self.L / Nv, Nv)
        g = np.meshgrid(c0, c0, c0, indexing='ij')
        self.cv = np.stack([x.ravel() for x in g])
        qz, qw = gauss_jacobi(self.Nrho, 0., 0.)
        self.qz = (self.R / 2.0) * (1.0 + qz)
        self.qw = ((self.R - 0.0) / 2.0) * qw
        self.M = M
        self.sz = sphere_design(M)
        self.sw = 4 * np.pi / M


def vhs_prefactor(vm, omega, dRef, Tref, alpha=1.0):
    """invKn and prefactor of the VHS model (std/scattering.py:70-83)."""
    invKn = (vm.H0 * np.sqrt(2.0) * np.pi * vm.n0 * dRef * dRef
             * pow(Tref / vm.T0, omega - 0.5))
    prefac = invKn * alpha / (pow(2.0, 2 - omega + alpha)
                              * math.gamma(2.5 - omega) * np.pi)
    return invKn, prefac


def vss_prefactor(vm, p, q, alpha, omega, dRef, Tref):
    """Pair prefactor of the VSS mixture model (bi/scattering.py:66-89)."""
    m = vm.masses
    invKn = (np.sqrt(1. + m[p] / m[q]) * np.pi * vm.n0 * dRef * dRef
             * pow(Tref / vm.T0, omega - 0.5) * vm.H0)
    mu = m[p] * m[q] / (m[p] + m[q])
    prefac = invKn * alpha / (np.sqrt(1. + m[p] / m[q]) * pow(mu, omega - 0.5)
                              * pow(2., 1 + alpha) * math.gamma(2.5 - omega)
                              * np.pi)
    return invKn, prefac


def fft_lvectors(N):
    """Integer wave numbers in FFT order, x slowest (std/scattering.py:116-128)."""
    l0 = np.concatenate((np.arange(0, N // 2), np.arange(-N // 2, 0)))
    g = np.meshgrid(l0, l0, l0, indexing='ij')
    return np.stack([x.ravel() for x in g]).astype(np.float64)
