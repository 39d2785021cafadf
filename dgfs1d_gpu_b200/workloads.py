"""Seeded synthetic workloads of the benchmark configurations.

Distributions are Maxwellians f = rho/(pi T)^{3/2} exp(-|c-u|^2/T)
(dgfs1D/std/initcond.py:58-60) with seeded bulk velocity / temperature
profiles, times (1 + eps U[-1,1]) i.i.d. noise per phase-space point.
"""
import math

import numpy as np

from .quadrature import gauss_jacobi
from .sphericaldesign import get_sphquadrule

SEED = 20261203


def vhs_mesh_params(N, M, Nrho, dev, full_sphere, omega=0.81, dRef=4.17e-10,
                    Tref=273., T0=273., H0=1e-3, rho0=1e-4,
                    molarMass0=39.96e-3, cmax=0.0, Tmax=273.):
    """Velocity-mesh and VHS parameters (std/velocitymesh.py:24-105,
    std/scattering.py:70-83) from explicit values."""
    NA, R0 = 6.0221409e+23, 8.3144598
    n0 = rho0 / molarMass0 * NA
    u0 = math.sqrt(2 * R0 / molarMass0 * T0)
    L = cmax / u0 + dev * math.sqrt(Tmax / T0)
    R = 2 * (L * 2.0 / (3.0 + math.sqrt(2.0)))
    z, w = gauss_jacobi(Nrho, 0., 0.)
    qz, qw = (R / 2.0) * (1.0 + z), (R / 2.0) * w
    if full_sphere:
        sz = get_sphquadrule('symmetric', 'womersley', npts=M).pts
        sw, sf = 4 * math.pi / M, 1.0
    else:
        sz = get_sphquadrule('symmetric', 'womersley', npts=2 * M).pts[:M]
        sw, sf = 2 * math.pi / M, 2.0
    invKn = H0 * math.sqrt(2.0) * math.pi * n0 * dRef * dRef \
        * (Tref / T0) ** (omega - 0.5)
    prefac = invKn / (2.0 ** (2 - omega + 1.0) * math.gamma(2.5 - omega)
                      * math.pi)
    c0 = np.linspace(-L + L / N, L - L / N, N)
    return dict(N=N, L=L, qz=qz, qw=qw, sz=sz, sw=sw, sphere_factor=sf,
                gamma=2.0 * (1 - omega), prefac=prefac, cw=(2.0 * L / N) ** 3,
                c0=c0)


def couette_distributions(c0, nslots, noise=0.01, seed=SEED):
    """Maxwellians with u_y in [-0.1, 0.1], T in [0.95, 1.05], perturbed."""
    rng = np.random.default_rng(seed)
    g = np.meshgrid(c0, c0, c0, indexing='ij')
    cx, cy, cz = (x.ravel() for x in g)
    f = np.empty((nslots, len(cx)))
    for s in range(nslots):
        uy = rng.uniform(-0.1, 0.1)
        T = rng.uniform(0.95, 1.05)
        m = np.exp(-(cx ** 2 + (cy - uy) ** 2 + cz ** 2) / T) \
            / (np.pi * T) ** 1.5
        f[s] = m * (1 + noise * rng.uniform(-1, 1, m.shape))
    return f
