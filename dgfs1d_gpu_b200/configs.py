"""INI texts of the benchmark / test configurations (nondimensional setups
expressed in the reference's dimensional INI keys)."""
import math

NA, R0 = 6.0221409e+23, 8.3144598


def rho0_for_knudsen(Kn, H0=1e-3, dRef=4.17e-10, omega=0.81, Tref=273.,
                     T0=273., molarMass0=39.96e-3):
    """rho0 giving invKn = 1/Kn in std/scattering.py:77-78."""
    n0 = (1.0 / Kn) / (H0 * math.sqrt(2.0) * math.pi * dRef * dRef
                        * (Tref / T0) ** (omega - 0.5))
    return n0 * molarMass0 / NA


def couette_std_ini(Ne=4, K=3, Nv=16, Nrho=8, M=6, dev=5.0, Kn=0.1,
                    omega=0.81, uwall=0.1, scheme='euler', dt=0.00025,
                    nsteps=52, precision='double', basis='nodal-sem-gll',
                    noise=0.01, seed=20261203, precision_mode=None,
                    sphere='auto', ic='maxwellian-noise'):
    T0, molarMass0 = 273., 39.96e-3
    u0 = math.sqrt(2 * R0 / molarMass0 * T0)
    rho0 = rho0_for_knudsen(Kn, omega=omega)
    pm = f'precision-mode = {precision_mode}\n' if precision_mode else ''
    return f"""
[config]
precision = {precision}
[mesh]
xlo = 0.
xhi = 1e-3
Ne = {Ne}
H0 = 1e-3
[basis]
kind = {basis}
K = {K}
Nqr = {K}
[non-dim]
T0 = {T0}
rho0 = {rho0!r}
molarMass0 = {molarMass0}
[velocity-mesh]
Nv = {Nv}
Nrho = {Nrho}
dev = {dev}
cmax = 0
Tmax = {T0}
[spherical-design-rule]
ssrule = womersley
M = {M}
sphere = {sphere}
[scattering-model]
type = vhs-gll
omega = {omega}
dRef = 4.17e-10
Tref = 273
muRef = 2.117e-5
{pm}
[time-integrator]
scheme = {scheme}
controller = none
tstart = 0.0
tend = {dt * nsteps!r}
dt = {dt!r}
[soln-ics]
type = {ic}
rho = {rho0!r}
T = {T0}
ux = 0
uy = 0
uz = 0
noise = {noise}
seed = {seed}
[soln-bcs-xlo]
type = dgfs-wall-diffuse
T = {T0}
ux = 0
uy = {-uwall * u0!r}
uz = 0
[soln-bcs-xhi]
type = dgfs-wall-diffuse
T = {T0}
ux = 0
uy = {uwall * u0!r}
uz = 0
"""


def couette_c2_ini(precision_mode='fp32', nsteps=200, Ne=8, K=3, Nv=32,
                   Nrho=16, M=12, dev=6.0, scheme='ssp-rk3', noise=0.01,
                   seed=20261203):
    """The batched FP32 Couette configuration: Ne=8, K=3 (24 points),
    N=32 on [-6, 6]^3, the full 12-point design, Nrho=16, ssp-rk3, diffuse
    walls at T=1 with u_y = -+0.1; initial Maxwellian (nondimensional) with
    u_y linear from -0.1 to 0.1 across the slab and T linear from 0.95 to
    1.05, times (1 + 0.01 U[-1, 1]) seeded noise; dt = 0.001/Ne as for the
    12-point configuration (whose 52 Euler steps use 0.001/4)."""
    ini = couette_std_ini(Ne=Ne, K=K, Nv=Nv, Nrho=Nrho, M=M, dev=dev,
                          scheme=scheme, dt=0.001 / Ne, nsteps=nsteps,
                          precision_mode=precision_mode, sphere='full')
    head, rest = ini.split('[soln-ics]', 1)
    tail = rest[rest.index('[soln-bcs-xlo]'):]
    ics = f"""[soln-ics]
type = maxwellian-expr-nondim
rho = 1.0
ux = 0.0
uy = -0.1 + 0.2*x
uz = 0.0
T = 0.95 + 0.1*x
noise = {noise}
seed = {seed}
"""
    return head + ics + tail


def couette_bi_ini(Ne=3, K=3, Nv=8, Nrho=4, M=6, Mpre=12, dev=5.0,
                   scheme='euler', dt=0.0005, nsteps=3, uwall=0.1,
                   noise=0.02, seed=20261203, compat=0,
                   masses=(39.96e-3, 83.77e-3), precision_mode=None):
    """Binary Couette (examples/bi/couette/dgfs1D.ini parameters, small).
    ``precision_mode`` ('fp64'/'fp32') sets [scattering-model] precision-mode."""
    pm = '' if precision_mode is None else f'precision-mode = {precision_mode}'
    T0, m0 = 273., masses[0]
    u0 = math.sqrt(2 * R0 / m0 * T0)
    rho0 = 0.00011140244750324529
    n0 = rho0 / m0 * NA
    return f"""
[config]
precision = double
[mesh]
xlo = 0.
xhi = 1e-3
Ne = {Ne}
H0 = 1e-3
[basis]
kind = nodal-sem-gll
K = {K}
Nqr = {K}
[non-dim]
T0 = {T0}
rho0 = {rho0!r}
molarMass0 = {m0}
[velocity-mesh]
nspcs = 2
Nv = {Nv}
Nrho = {Nrho}
dev = {dev}
cmax = 0
Tmax = {T0}
molarMass1 = {masses[0]}
molarMass2 = {masses[1]}
[spherical-design-rule]
ssrule = womersley
M = {M}
[scattering-model]
type = vss
ssrulepre = womersley
Mpre = {Mpre}
{pm}
alpha00 = 1.4
omega00 = 0.81
dRef00 = 4.11e-10
Tref00 = 273
alpha01 = 1.36
omega01 = 0.805
dRef01 = 4.405e-10
Tref01 = 273
alpha10 = 1.36
omega10 = 0.805
dRef10 = 4.405e-10
Tref10 = 273
alpha11 = 1.32
omega11 = 0.80
dRef11 = 4.7e-10
Tref11 = 273
[time-integrator]
scheme = {scheme}
tstart = 0.0
tend = {dt * nsteps!r}
dt = {dt!r}
bi-ssp-rk3-compat = {compat}
[soln-ics]
type = maxwellian-noise
nden1 = {0.5 * n0!r}
nden2 = {0.5 * n0!r}
T = {T0}
ux = 0
uy = 0
uz = 0
noise = {noise}
seed = {seed}
[soln-bcs-xlo]
type = dgfs-wall-diffuse
T = {T0}
ux = 0
uy = {-uwall * u0!r}
uz = 0
[soln-bcs-xhi]
type = dgfs-wall-diffuse
T = {T0}
ux = 0
uy = {uwall * u0!r}
uz = 0
"""


def couette_astd_ini(scheme='imex-lm-bdf2', penalty='boltz-bgk-direct-gll',
                     dt=0.002, nsteps=3, **kw):
    """The Couette set-up of couette_std_ini with a penalty model and an IMEX
    scheme (dgfsABstd1D keys)."""
    ini = couette_std_ini(scheme=scheme, dt=dt, nsteps=nsteps, **kw)
    return ini + """
[penalized-scattering-model]
type = {0}
omega = 0.81
muRef = 2.117e-5
Tref = 273
""".format(penalty)


def normal_shock_std_ini(Mach=1.5, Ne=32, K=3, Nv=48, Nrho=24, M=32, dev=8.0,
                         omega=0.5, scheme='lse-rk45', dt=None, nsteps=500,
                         half_width=20.0, ramp=2.0, noise=0.005,
                         seed=20261203, precision_mode='fp32', sphere='full',
                         basis='nodal-sem-gll'):
    """Normal shock of a monatomic hard-sphere gas: Rankine-Hugoniot states
    at Mach `Mach` (gamma = 5/3), joined by a tanh ramp of width `ramp` mean
    free paths on x in [-half_width, half_width] mean free paths (the mean
    free path is the reference length H0, Kn = 1), with inlet boundaries at
    both ends and (1 + noise U[-1, 1]) seeded noise."""
    g = 5.0 / 3.0
    T0, molarMass0 = 273., 39.96e-3
    H0 = 1e-3
    rho1 = rho0_for_knudsen(1.0, H0=H0, omega=omega)
    R = R0 / molarMass0
    u1 = Mach * math.sqrt(g * R * T0)
    r = (g + 1) * Mach ** 2 / ((g - 1) * Mach ** 2 + 2)
    tr = ((2 * g * Mach ** 2 - (g - 1)) * ((g - 1) * Mach ** 2 + 2)
          / ((g + 1) ** 2 * Mach ** 2))
    rho2, T2, u2 = rho1 * r, T0 * tr, u1 / r
    u0 = math.sqrt(2 * R0 / molarMass0 * T0)
    if dt is None:
        # advective CFL of the nodal DG scheme on the finest node spacing
        dx = 2 * half_width / Ne / (K * K)
        dt = 0.5 * dx / (dev + u1 / u0)
    pm = f'precision-mode = {precision_mode}\n' if precision_mode else ''
    return f"""
[config]
precision = double
[mesh]
xlo = {-half_width * H0!r}
xhi = {half_width * H0!r}
Ne = {Ne}
H0 = {H0}
[basis]
kind = {basis}
K = {K}
Nqr = {K}
[non-dim]
T0 = {T0}
rho0 = {rho1!r}
molarMass0 = {molarMass0}
[velocity-mesh]
Nv = {Nv}
Nrho = {Nrho}
dev = {dev}
cmax = 0
Tmax = {T0}
[spherical-design-rule]
ssrule = womersley
M = {M}
sphere = {sphere}
[scattering-model]
type = vhs-gll
omega = {omega}
dRef = 4.17e-10
Tref = 273
muRef = 2.117e-5
{pm}
[time-integrator]
scheme = {scheme}
controller = none
tstart = 0.0
tend = {dt * nsteps!r}
dt = {dt!r}
[soln-ics]
type = normal-shock
rho1 = {rho1!r}
T1 = {T0}
ux1 = {u1!r}
rho2 = {rho2!r}
T2 = {T2!r}
ux2 = {u2!r}
x0 = 0.0
width = {ramp * H0!r}
noise = {noise}
seed = {seed}
[soln-bcs-xlo]
type = dgfs-inlet
rho = {rho1!r}
T = {T0}
ux = {u1!r}
uy = 0
uz = 0
[soln-bcs-xhi]
type = dgfs-inlet
rho = {rho2!r}
T = {T2!r}
ux = {u2!r}
uy = 0
uz = 0
"""


def sod_astd_ini(Ne=8, K=3, Nv=32, Nrho=6, M=6, dev=7.0, dt=1e-3, nsteps=10,
                 scheme='imex-lm-bdf1', penalty='boltz-shakov-direct-gll',
                 limiter=1, sphere='auto'):
    """Sod shock tube of nitrogen-like gas on [-5, 5] (mean free paths) for
    dgfsABstd1D: the set-up of the reference's abstd sod example (the keys
    and physical values it uses: inlet walls at the two states, VHS
    omega = 0.77 Boltzmann operator, Shakov penalty, IMEX-LM BDF1, slope
    limiter), at a chosen resolution."""
    T0, rho0, m0 = 278.746, 125e-9, 28.96278e-3
    return f"""
[config]
precision = double
[mesh]
xlo = -5
xhi = 5
Ne = {Ne}
H0 = 1
[basis]
kind = nodal-sem-gll
K = {K}
Nq = {K}
Nqr = 16
[non-dim]
T0 = {T0}
rho0 = {rho0}
molarMass0 = {m0}
[velocity-mesh]
Nv = {Nv}
Nrho = {Nrho}
dev = {dev}
cmax = 0
Tmax = 348.4
[spherical-design-rule]
ssrule = womersley
M = {M}
sphere = {sphere}
[penalized-scattering-model]
type = {penalty}
omega = 0.81
muRef = 2.117e-5
Tref = 273
[scattering-model]
type = vhs-gll
omega = 0.77
muRef = 1.7175337355197123e-05
dRef = 4.19e-10
Tref = 273
[time-integrator]
scheme = {scheme}
controller = none
tstart = 0.0
tend = {dt * nsteps!r}
dt = {dt!r}
limiter = {limiter}
[soln-ics]
type = sod-shock-tube
rho-left = 1000e-9
T-left = 348.432
rho-right = 125e-9
T-right = 278.746
[soln-bcs-xlo]
type = dgfs-inlet
T = 348.432
ux = 0
uy = 0
uz = 0
rho = 1000e-9
[soln-bcs-xhi]
type = dgfs-inlet
T = 278.746
ux = 0
uy = 0
uz = 0
rho = 125e-9
"""
