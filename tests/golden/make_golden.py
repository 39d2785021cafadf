"""Generate the golden vectors of tests/golden from the reference itself.

Run in a container where the reference checkout exists, with ``$DGFS_REF``
set to it (the directory that holds dgfs1D/)::

    python tests/golden/make_golden.py
    python tests/golden/make_golden.py penalty-models   # only the ES-BGK/Shakov files
    python tests/golden/make_golden.py limiter          # only the slope-limiter file
    python tests/golden/make_golden.py moments          # only the moment-writer file
    python tests/golden/make_golden.py upwind           # only the upwind (abstdu) file
    python tests/golden/make_golden.py std-relax        # only the dgfsStd1D relaxation file
    python tests/golden/make_golden.py penalty          # only the BGK penalty-kernel file
    python tests/golden/make_golden.py entropy          # only the entropy-stable (abstde2) file

What runs from the reference:
  * its pure-Python setup code, imported directly with stand-ins for the
    GPU/MPI packages it imports but that this setup does not use (pycuda,
    mpi4py, gimmik, the cuFFT/cuBLAS ctypes bindings): quadratures,
    spherical-design loading, velocity meshes, the VHS/VSS prefactors
    (load_parameters) and the nodal DG bases;
  * its Mako CUDA kernels, rendered and compiled for the CPU by
    ``oracle/ref_build.py``, driven in the exact call sequence of
    ``DGFSVHSGLLScatteringModelStd.fs``, ``DGFSVHSScatteringModelStd.fs`` and
    ``DGFSBiVSSScatteringModel.fs``; the cuFFT calls of those sequences are
    replaced by pocketfft with cuFFT's conventions (cuFFT is a closed library
    with no CPU build).

Inputs are seeded; outputs are written as small .npz files beside this script.
"""
import configparser
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF = os.environ.get('DGFS_REF')
SEED = 20261203


# -- stand-ins for modules the setup code imports but does not use -----------

def _install_stubs():
    def mod(name, **attrs):
        m = types.ModuleType(name)
        m.__dict__.update(attrs)
        sys.modules[name] = m
        return m

    class _Arr(np.ndarray):
        pass

    def to_gpu(a):
        return np.asarray(a)

    gpuarray = mod('pycuda.gpuarray', to_gpu=to_gpu, empty=np.empty,
                   zeros=np.zeros, empty_like=np.empty_like,
                   GPUArray=np.ndarray)
    compiler = mod('pycuda.compiler', SourceModule=lambda *a, **k: None)
    driver = mod('pycuda.driver', func_cache=types.SimpleNamespace(
        PREFER_L1=None), memcpy_dtod=lambda *a: None)
    mod('pycuda', gpuarray=gpuarray, compiler=compiler, driver=driver)

    class _Comm:
        rank, size = 0, 1

        def Get_rank(self):
            return 0

        def Get_size(self):
            return 1

    mpi = types.SimpleNamespace(COMM_WORLD=_Comm(), PROC_NULL=-1)
    mod('mpi4py', MPI=mpi, rc=types.SimpleNamespace(initialize=False))
    mod('mpi4py.MPI', COMM_WORLD=mpi.COMM_WORLD, PROC_NULL=-1)
    mod('mpi4py.rc', initialize=False)
    mod('gimmik', generate_mm=lambda *a, **k: '')

    class _Lookup:
        def __init__(self, *a, **k):
            pass

    class _Template:
        def __init__(self, *a, **k):
            pass

    mako = mod('mako')
    mako.lookup = mod('mako.lookup', TemplateLookup=_Lookup)
    mako.template = mod('mako.template', Template=_Template)
    for name in ('cufft', 'cublas', 'cusolver', 'cusparse'):
        m = mod('dgfs1D.' + name)
        m.__getattr__ = lambda attr: (lambda *a, **k: None)
    # Python 3.12 removed the deprecated alias the reference imports
    configparser.SafeConfigParser = configparser.ConfigParser


def _import_reference():
    if not REF:
        raise SystemExit('set DGFS_REF to the reference checkout (the '
                         'directory that holds dgfs1D/)')
    _install_stubs()
    sys.path.insert(0, REF)
    import dgfs1D.nputil as nputil
    nputil.get_comm_rank_root = lambda: (sys.modules['mpi4py'].MPI.COMM_WORLD,
                                         0, 0)
    from dgfs1D import quadratures, basis, dictionary  # noqa: F401
    import dgfs1D.util as util
    util.get_mm_kernel = lambda *a, **k: None
    import dgfs1D.basis as basis
    basis.get_mm_kernel = lambda *a, **k: None
    from dgfs1D.std import velocitymesh as vstd
    from dgfs1D.bi import velocitymesh as vbi
    from dgfs1D.std import scattering as sstd
    from dgfs1D.bi import scattering as sbi
    # the module re-binds the class name DGFSVHSGLLScatteringModelStd later
    # (std/scattering.py:708-741); resolve the model as the drivers do
    vhsgll = nputil.subclass_where(sstd.DGFSScatteringModelStd,
                                   scattering_model='vhs-gll')
    return types.SimpleNamespace(quadratures=quadratures, basis=basis,
                                 Dictionary=dictionary.Dictionary, vstd=vstd,
                                 vbi=vbi, sstd=sstd, sbi=sbi, VHSGLL=vhsgll)


STD_INI = """
[config]
precision = double
[mesh]
xlo = 0.
xhi = 1e-3
Ne = 4
H0 = 1e-3
[basis]
kind = {basis}
K = 3
Nqr = 8
[non-dim]
T0 = 273
rho0 = 0.00023
molarMass0 = 39.96e-3
[velocity-mesh]
Nv = {Nv}
Nrho = {Nrho}
dev = {dev}
cmax = 0
Tmax = 273
[spherical-design-rule]
ssrule = womersley
M = {M}
[scattering-model]
type = vhs-gll
omega = 0.81
dRef = 4.17e-10
Tref = 273
muRef = 2.117e-5
"""

BI_INI = """
[config]
precision = double
[mesh]
xlo = 0.
xhi = 1e-3
Ne = 2
H0 = 1e-3
[non-dim]
T0 = 273
rho0 = 0.00011140244750324529
molarMass0 = 39.96e-3
[velocity-mesh]
nspcs = 2
Nv = {Nv}
Nrho = {Nrho}
dev = {dev}
cmax = 0
Tmax = 273
molarMass1 = 39.96e-3
molarMass2 = 83.77e-3
[spherical-design-rule]
ssrule = womersley
M = {M}
[scattering-model]
type = vss
ssrulepre = womersley
Mpre = {Mpre}
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
"""


def _fwd(x):
    """CUFFT_FORWARD on the last three axes (batched like cufftPlanMany)."""
    return np.fft.fftn(x, axes=(-3, -2, -1))


def _inv(x):
    """CUFFT_INVERSE (unnormalised) on the last three axes."""
    n = x.shape[-1] * x.shape[-2] * x.shape[-3]
    return np.fft.ifftn(x, axes=(-3, -2, -1)) * n


def _maxwellian_noise(cv, rng, rho=1.0, noise=0.02):
    uy, T = rng.uniform(-0.1, 0.1), rng.uniform(0.9, 1.1)
    m = rho * np.exp(-(cv[0] ** 2 + (cv[1] - uy) ** 2 + cv[2] ** 2) / T) \
        / (np.pi * T) ** 1.5
    return m * (1 + noise * rng.uniform(-1, 1, m.shape))


def golden_vhs(R, Nv=8, Nrho=4, M=6, dev=5.0, Ne=3):
    """Reference kernels of vhs-gll / vhs, driven like fs()."""
    from oracle.ref_build import RefModule, grid_for, render_template
    cfg = R.Dictionary(STD_INI.format(basis='nodal-sem-gll', Nv=Nv,
                                      Nrho=Nrho, M=M, dev=dev))
    vm = R.vstd.DGFSVelocityMeshStd(cfg)
    sm = object.__new__(R.VHSGLL)
    sm.cfg, sm.vm, sm._Ne = cfg, vm, Ne
    sm.load_parameters()
    vsize, N = vm.vsize(), vm.Nv()
    l0 = np.concatenate((np.arange(0, N / 2), np.arange(-N / 2, 0)))
    l = np.zeros((3, vsize))
    for idv in range(vsize):
        l[0, idv] = l0[idv // (N * N)]
        l[1, idv] = l0[(idv % (N * N)) // N]
        l[2, idv] = l0[(idv % (N * N)) % N]
    src = render_template(
        'dgfs1D/std/kernels/scattering/vhs-gll.mako', dtype='double',
        Nrho=Nrho, M=vm.M(), vsize=vsize, sw=vm.sw(), prefac=sm._prefactor,
        qw=vm.qw(), sz=vm.sz(), gamma=sm._gamma, L=vm.L(), qz=vm.qz(),
        Ne=Ne, block_size=128, cw=vm.cw())
    K = RefModule(src, tag='vhs-gll')
    blk = 128
    g = grid_for(vsize, blk)
    lx, ly, lz = (np.ascontiguousarray(l[i]) for i in range(3))
    aa = np.empty(Nrho * M * vsize)
    K.launch('precompute_aa', g, blk, lx, ly, lz, aa)
    bb1, bb2 = np.empty(Nrho * vsize), np.empty(vsize)
    K.launch('precompute_bb', g, blk, lx, ly, lz, bb1, bb2)

    rng = np.random.default_rng(SEED)
    Kb = 2  # modes
    f = np.stack([_maxwellian_noise(vm.cv(), rng) for _ in range(Kb * Ne)])
    gfun = np.stack([_maxwellian_noise(vm.cv(), rng) for _ in range(Kb * Ne)])
    f = np.ascontiguousarray(f.ravel())
    gfun = np.ascontiguousarray(gfun.ravel())

    def cplx(n):
        return np.zeros(n, dtype=np.complex128)

    shape = (N, N, N)
    Qgll = np.zeros(Kb * Ne * vsize)
    Qvhs = np.zeros(Kb * Ne * vsize)
    for m in range(Kb):
        for e in range(Ne):
            # DGFSVHSGLLScatteringModelStd.fs (std/scattering.py:251-313)
            fC = cplx(vsize)
            K.launch('r2z_', g, blk, e, m, f, fC)
            FTf = _fwd(fC.reshape(shape)).ravel()
            t1, t2 = cplx(Nrho * M * vsize), cplx(Nrho * M * vsize)
            K.launch('cosSinMul', g, blk, aa, FTf, t1, t2)
            t3 = _inv(t1.reshape(-1, *shape)).ravel()
            t4 = _inv(t2.reshape(-1, *shape)).ravel()
            K.launch('magSqr', g, blk, t3, t4, t2)
            t1 = _fwd(t2.reshape(-1, *shape)).ravel()
            K.launch('computeQG', g, blk, bb1, t1, fC)
            QG = _inv(fC.reshape(shape)).ravel()
            K.launch('ax', g, blk, bb2, FTf)
            fC = _inv(FTf.reshape(shape)).ravel()
            K.launch('output_append_', g, blk, e, m, m, QG, fC, f, Qgll)
            # DGFSVHSScatteringModelStd.fs (std/scattering.py:346-429)
            fC, gC = cplx(vsize), cplx(vsize)
            K.launch('r2z_', g, blk, e, m, f, fC)
            K.launch('r2z_', g, blk, e, m, gfun, gC)
            FTf = _fwd(fC.reshape(shape)).ravel()
            FTg = _fwd(gC.reshape(shape)).ravel()
            t1, t2 = cplx(Nrho * M * vsize), cplx(Nrho * M * vsize)
            K.launch('cosMul', g, blk, aa, FTf, FTg, t1, t2)
            t3 = _inv(t1.reshape(-1, *shape)).ravel()
            t4 = _inv(t2.reshape(-1, *shape)).ravel()
            t5 = cplx(Nrho * M * vsize)
            K.launch('cplxMul', g, blk, t3, t4, t5)
            K.launch('sinMul', g, blk, aa, FTf, FTg, t1, t2)
            t3 = _inv(t1.reshape(-1, *shape)).ravel()
            t4 = _inv(t2.reshape(-1, *shape)).ravel()
            K.launch('cplxMulAdd', g, blk, t3, t4, t5)
            t1 = _fwd(t5.reshape(-1, *shape)).ravel()
            fC = cplx(vsize)
            K.launch('computeQG', g, blk, bb1, t1, fC)
            QG = _inv(fC.reshape(shape)).ravel()
            K.launch('ax', g, blk, bb2, FTg)
            fC = _inv(FTg.reshape(shape)).ravel()
            K.launch('output_append_', g, blk, e, m, m, QG, fC, f, Qvhs)
    return dict(Nv=Nv, Nrho=Nrho, M=M, Ne=Ne, L=vm.L(), qz=vm.qz(),
                qw=vm.qw(), sz=vm.sz(), sw=vm.sw(), cw=vm.cw(), cv=vm.cv(),
                prefac=sm._prefactor, gamma=sm._gamma, aa=aa, bb1=bb1,
                bb2=bb2, f=f, g=gfun, Q_vhs_gll=Qgll, Q_vhs=Qvhs,
                prefacBGK=sm._prefactorBGK)


def golden_vss(R, Nv=8, Nrho=4, M=6, Mpre=12, dev=5.0, Ne=2):
    """Reference kernels of vss, driven like DGFSBiVSSScatteringModel.fs."""
    from oracle.ref_build import RefModule, grid_for, render_template
    cfg = R.Dictionary(BI_INI.format(Nv=Nv, Nrho=Nrho, M=M, Mpre=Mpre,
                                     dev=dev))
    vm = R.vbi.DGFSVelocityMeshBi(cfg)
    sm = object.__new__(R.sbi.DGFSBiVSSScatteringModel)
    sm.cfg, sm.vm, sm._Ne, sm._nspcs = cfg, vm, Ne, vm.nspcs()
    sm.load_parameters()
    vsize, N = vm.vsize(), vm.Nv()
    l0 = np.concatenate((np.arange(0, N / 2, dtype=np.int32),
                         np.arange(-N / 2, 0, dtype=np.int32)))
    l = np.zeros((3, vsize), dtype=np.int32)
    for idv in range(vsize):
        l[0, idv] = l0[idv // (N * N)]
        l[1, idv] = l0[(idv % (N * N)) // N]
        l[2, idv] = l0[(idv % (N * N)) % N]
    sz, qz, qw, sw = vm.sz(), vm.qz(), vm.qw(), vm.sw()
    src = render_template(
        'dgfs1D/bi/kernels/scattering/vss.mako', dtype='double', Nrho=Nrho,
        M=M, vsize=vsize, sw=sw, prefac=sm._prefactor, cases=sm._cases,
        masses=vm.masses(), qw=qw, qz=qz, L=vm.L(), sz=sz, gamma=sm._gamma,
        eta=sm._eta, Mpre=sm._Mpre, szpre=sm._szpre, swpre=sm._swpre)
    K = RefModule(src, tag='vss')
    blk = 256
    g = grid_for(vsize, blk)
    lx, ly, lz = (np.ascontiguousarray(l[i]) for i in range(3))
    aa = np.empty(Nrho * M * vsize)
    K.launch('precompute_a', g, blk, lx, ly, lz, aa)
    szx, szy, szz = (np.ascontiguousarray(sz[:, i]) for i in range(3))
    bb, cc = {}, {}
    for cp, cq in sm._cases:
        pq = f'{cp}{cq}'
        bb[pq] = np.empty(Nrho * M * vsize, dtype=np.complex128)
        cc[pq] = np.zeros(vsize, dtype=np.complex128)
        for p in range(Nrho):
            fac = np.pi / vm.L() * qz[p]
            fac_b = sm._swpre * pow(qz[p], sm._gamma[pq] + 2)
            fac_c = qw[p] * sw * fac_b
            for q in range(M):
                K.launch('precompute_bc_' + pq, g, blk, p, q, float(fac),
                         float(fac_b), float(fac_c), lx, ly, lz, szx, szy,
                         szz, bb[pq], cc[pq])
    rng = np.random.default_rng(SEED + 1)
    Kb = 2
    fs = []
    for sp in range(2):
        rho = [0.5, 0.5][sp]
        fs.append(np.ascontiguousarray(np.stack(
            [_maxwellian_noise(vm.cv(), rng, rho=rho) for _ in range(Kb * Ne)]
        ).ravel()))
    shape = (N, N, N)

    def cplx(n):
        return np.zeros(n, dtype=np.complex128)

    Q = {pq: np.zeros(Kb * Ne * vsize) for pq in bb}
    for cp, cq in sm._cases:
        pq = f'{cp}{cq}'
        for m in range(Kb):
            for e in range(Ne):
                f1C, f2C = cplx(vsize), cplx(vsize)
                K.launch('r2z', g, blk, Ne, e, m, fs[cp], f1C)
                K.launch('r2z', g, blk, Ne, e, m, fs[cq], f2C)
                FTf = _fwd(f1C.reshape(shape)).ravel()
                FTg = _fwd(f2C.reshape(shape)).ravel()
                t1, t2 = cplx(Nrho * M * vsize), cplx(Nrho * M * vsize)
                K.launch('cosSinMul_' + pq, g, blk, aa, FTf, FTg, t1, t2)
                t3 = _inv(t1.reshape(-1, *shape)).ravel()
                t1 = _inv(t2.reshape(-1, *shape)).ravel()
                K.launch('prod', g, blk, t3, t1, t2)
                t1 = _fwd(t2.reshape(-1, *shape)).ravel()
                # computeQG writes QG[idx] also for idx >= vsize
                # (vss.mako:240); give it a grid-sized buffer
                QGh = cplx(g * blk)
                K.launch('computeQG', g, blk, bb[pq], t1, QGh)
                QG = _inv(QGh[:vsize].reshape(shape)).ravel()
                K.launch('ax2', g, blk, cc[pq], FTg, FTf)
                f2C = _inv(FTf.reshape(shape)).ravel()
                K.launch('output_' + pq, g, blk, Ne, e, m, m, QG, f2C,
                         fs[cp], Q[pq])
    out = dict(Nv=Nv, Nrho=Nrho, M=M, Mpre=Mpre, Ne=Ne, L=vm.L(),
               qz=qz, qw=qw, sz=sz, sw=sw, szpre=sm._szpre, cw=vm.cw(),
               cv=vm.cv(), masses=np.array(vm.masses()), f0=fs[0], f1=fs[1],
               aa=aa)
    for pq in bb:
        out['prefac' + pq] = sm._prefactor[pq]
        out['gamma' + pq] = sm._gamma[pq]
        out['eta' + pq] = sm._eta[pq]
        out['b' + pq] = bb[pq]
        out['c' + pq] = cc[pq]
        out['Q' + pq] = Q[pq]
    return out


def _vhs_ref_fs(R, cfg, vm, Ne, Kb):
    """fs(f_slots, Q_slots, e, m) driving the reference vhs-gll kernels."""
    from oracle.ref_build import RefModule, grid_for, render_template
    sm = object.__new__(R.VHSGLL)
    sm.cfg, sm.vm, sm._Ne = cfg, vm, Ne
    sm.load_parameters()
    vsize, N, Nrho, M = vm.vsize(), vm.Nv(), vm.Nrho(), vm.M()
    l0 = np.concatenate((np.arange(0, N / 2), np.arange(-N / 2, 0)))
    l = np.zeros((3, vsize))
    for idv in range(vsize):
        l[0, idv] = l0[idv // (N * N)]
        l[1, idv] = l0[(idv % (N * N)) // N]
        l[2, idv] = l0[(idv % (N * N)) % N]
    src = render_template(
        'dgfs1D/std/kernels/scattering/vhs-gll.mako', dtype='double',
        Nrho=Nrho, M=M, vsize=vsize, sw=vm.sw(), prefac=sm._prefactor,
        qw=vm.qw(), sz=vm.sz(), gamma=sm._gamma, L=vm.L(), qz=vm.qz(),
        Ne=Ne, block_size=128, cw=vm.cw())
    K = RefModule(src, tag='vhs-gll')
    blk = 128
    g = grid_for(vsize, blk)
    lx, ly, lz = (np.ascontiguousarray(l[i]) for i in range(3))
    aa = np.empty(Nrho * M * vsize)
    K.launch('precompute_aa', g, blk, lx, ly, lz, aa)
    bb1, bb2 = np.empty(Nrho * vsize), np.empty(vsize)
    K.launch('precompute_bb', g, blk, lx, ly, lz, bb1, bb2)
    shape = (N, N, N)

    def fs(f, Q, e, r, m):
        fC = np.zeros(vsize, dtype=np.complex128)
        K.launch('r2z_', g, blk, e, r, f, fC)
        FTf = _fwd(fC.reshape(shape)).ravel()
        t1 = np.zeros(Nrho * M * vsize, dtype=np.complex128)
        t2 = np.zeros_like(t1)
        K.launch('cosSinMul', g, blk, aa, FTf, t1, t2)
        t3 = _inv(t1.reshape(-1, *shape)).ravel()
        t4 = _inv(t2.reshape(-1, *shape)).ravel()
        K.launch('magSqr', g, blk, t3, t4, t2)
        t1 = _fwd(t2.reshape(-1, *shape)).ravel()
        K.launch('computeQG', g, blk, bb1, t1, fC)
        QG = _inv(fC.reshape(shape)).ravel()
        K.launch('ax', g, blk, bb2, FTf)
        fC = _inv(FTf.reshape(shape)).ravel()
        K.launch('output_append_', g, blk, e, r, m, QG, fC, f, Q)
    return fs, sm


def golden_dg(R, kind, Nv=8, Nrho=4, M=6, dev=5.0, Ne=3, Kb=3):
    """One std.py rhs() through the reference's own std.mako and diffuse-wall
    kernels (+ the vhs-gll fs loop), on seeded data."""
    from oracle.ref_build import RefModule, grid_for, render_template
    ini = STD_INI.format(basis=kind, Nv=Nv, Nrho=Nrho, M=M, dev=dev)
    ini = ini.replace('Ne = 4', f'Ne = {Ne}').replace('K = 3', f'K = {Kb}')
    cfg = R.Dictionary(ini)
    vm = R.vstd.DGFSVelocityMeshStd(cfg)
    cls = {'nodal-sem-gll': R.basis.NodalSemGLL,
           'nodal-gll': R.basis.NodalGLL}[kind]
    basis = cls(cfg)
    K, Nqf, vsize = basis.K, basis.Nqf, vm.vsize()
    import dgfs1D.util as util
    xmesh = np.linspace(0., 1e-3, Ne + 1) / 1e-3
    h = np.diff(xmesh).reshape(-1, 1)
    jac, invjac = h / 2., 2. / h
    mapL, mapR = np.arange(Ne + 1) + (Nqf - 1) * Ne - 1, np.arange(Ne + 1)
    mapL[0], mapR[-1] = 0, Ne * Nqf - 1
    xsol = np.array([0.5 * (xmesh[j] + xmesh[j + 1]) + jac[j] * basis.z
                     for j in range(Ne)]).T
    src = render_template('dgfs1D/std/kernels/std.mako', K=K, Ne=Ne, Nq=K,
                          vsize=vsize, dtype='double', mapL=mapL, mapR=mapR,
                          offsetL=0, offsetR=len(mapR) - 1, invjac=invjac,
                          gRD=basis.gRD, gLD=basis.gLD, xsol=xsol)
    SK = RefModule(src, tag='std')
    walls = {}
    u0 = vm.u0()
    for side, nl, uy in (('L', -1., -0.1), ('R', 1., 0.1)):
        u_w = np.array([0., uy, 0.]).reshape(3, 1)
        T_w = 1.0
        f0 = ((1.0 / (np.pi * T_w) ** 1.5)
              * np.exp(-np.sum((vm.cv() - u_w) ** 2, axis=0) / T_w))
        bsrc = render_template('dgfs1D/std/kernels/bcs/dgfs-wall-diffuse.mako',
                               dtype='double', vsize=vsize, cw=vm.cw(),
                               ux=0.0, nl=nl, x=0.0)
        walls[side] = (RefModule(bsrc, tag='wall' + side), f0)
    blk = 128
    gv = grid_for(vsize, blk)
    filt = util.filter_tol

    def mm(A, B):
        return np.ascontiguousarray(
            (filt(np.array(A, dtype=np.float64)) @ B.reshape(A.shape[1], -1))
            .ravel())

    rng = np.random.default_rng(SEED + 7)
    u = np.stack([_maxwellian_noise(vm.cv(), rng, rho=1.0)
                  for _ in range(K * Ne)]).reshape(K, Ne, vsize)
    u = np.ascontiguousarray(u.ravel())
    fs, sm = _vhs_ref_fs(R, cfg, vm, Ne, K)
    out = {}
    for with_q in (False, True):
        usolF = mm(basis._Bqf.T, u)
        uL, uR = np.zeros((Ne + 1) * vsize), np.zeros((Ne + 1) * vsize)
        SK.launch('extract_left', gv, blk, usolF, uL)
        SK.launch('extract_right', gv, blk, usolF, uR)
        bcL, bcR, bcT = np.zeros(vsize), np.zeros(vsize), np.zeros(vsize)
        SK.launch('transfer_bc_left', gv, blk, uL, bcL)
        SK.launch('transfer_bc_right', gv, blk, uR, bcR)
        cvx = np.ascontiguousarray(vm.cv()[0])
        for side, bcv, ins in (('L', bcL, 'insert_bc_left'),
                               ('R', bcR, 'insert_bc_right')):
            BK, f0 = walls[side]
            num, den = np.zeros(vsize), np.zeros(vsize)
            BK.launch('updateBC', gv, blk, bcv, cvx, f0, num, den, 0.0)
            nden = np.array([-(np.sum(num) / np.sum(den))])
            BK.launch('applyBC', gv, blk, bcv, bcT, cvx, f0, nden, 0.0)
            SK.launch(ins, gv, blk, bcT, uL if side == 'L' else uR)
        jL, jR = np.zeros_like(uL), np.zeros_like(uR)
        SK.launch('flux', gv, blk, uL, uR, cvx, jL, jR)
        ux = mm(basis.derivMat, u)
        SK.launch('mul_by_adv', grid_for(K * Ne * vsize, blk), blk, cvx, ux)
        SK.launch('totalFlux', gv, blk, ux, cvx, jL, jR)
        SK.launch('mul_by_invjac', gv, blk, ux)
        if with_q:
            for m in range(K):
                d_f = mm(basis._U[m].T, u)
                d_g = mm(basis._V[m], u)
                for r in basis.sigModes[m]:
                    for e in range(Ne):
                        fs(d_f, ux, e, int(r), m)
        uout = mm(basis._B.T if kind == "nodal-sem-gll" else np.eye(K), ux)
        out['rhs_q' if with_q else 'rhs_adv'] = uout
    out.update(u=u, K=K, Ne=Ne, Nv=Nv, Nrho=Nrho, M=M, L=vm.L(), qz=vm.qz(),
               qw=vm.qw(), sz=vm.sz(), sw=vm.sw(), cw=vm.cw(), cv=vm.cv(),
               prefac=sm._prefactor, gamma=sm._gamma, invjac=invjac.ravel())
    return out


def golden_penalty(R, Nv=8, npts=6, omega=0.81, prefac=3.7):
    """The penalty kernels of astd bgk-direct-gll.mako on seeded data."""
    from oracle.ref_build import RefModule, grid_for, render_template
    vsize = Nv ** 3
    src = render_template(
        'dgfs1D/astd/kernels/scattering/bgk-direct-gll.mako', vsize=vsize,
        nalph=5, omega=omega, Pr=1.0, dtype='double', nbdf=[1, 2], nars=[1, 2])
    K = RefModule(src, tag='bgk')
    rng = np.random.default_rng(SEED + 11)
    L = 5.0
    c0 = np.linspace(-L + L / Nv, L - L / Nv, Nv)
    g = np.meshgrid(c0, c0, c0, indexing='ij')
    cv = np.stack([x.ravel() for x in g])
    cw = (2 * L / Nv) ** 3
    f = np.stack([_maxwellian_noise(cv, rng, rho=rng.uniform(0.5, 2))
                  for _ in range(npts)]).ravel()
    phi = np.vstack([np.ones(vsize), cv, np.sum(cv * cv, axis=0)]) * cw
    U = np.ascontiguousarray((f.reshape(npts, vsize) @ phi.T).ravel())
    blk = 256
    lda = npts * vsize
    gg = grid_for(lda, blk)
    cx, cy, cz = (np.ascontiguousarray(cv[i]) for i in range(3))
    M = np.zeros(lda)
    K.launch('cmaxwellian', gg, blk, lda, cx, cy, cz, M, U)
    Q = np.zeros(lda)
    K.launch('collide', gg, blk, prefac, lda, M, U, f, Q)
    out = dict(Nv=Nv, npts=npts, omega=omega, prefac=prefac, cv=cv, cw=cw,
               f=f, U=U, M=M, Q=Q)
    dt = 0.01
    L0 = rng.normal(size=lda) * 1e-3
    L1 = rng.normal(size=lda) * 1e-3
    f1 = f * (1 + 0.01 * rng.uniform(-1, 1, lda))
    LU0 = rng.normal(size=npts * 5) * 1e-3
    LU1 = rng.normal(size=npts * 5) * 1e-3
    U1 = U * (1 + 0.01 * rng.uniform(-1, 1, U.shape))
    Un = np.zeros(npts * 5)
    gm = grid_for(npts, blk)
    # bdf-222 coefficients, called as Bdf222IntegratorAstd does
    a1, a2, a3, g1, g2, b = 1. / 3., -4. / 3., 1., -2. / 3., 4. / 3., 2. / 3.
    K.launch('updateMom2_BDF', gm, blk, prefac, npts, dt, a1, U, -g1, LU0,
             a2, U1, -g2, LU1, a3, Un, b)
    fn = np.zeros(lda)
    K.launch('updateDistribution2_BDF', gg, blk, prefac, lda, dt, a1, f, -g1,
             L0, a2, f1, -g2, L1, b, M, a3, Un, fn)
    out.update(dt=dt, L0=L0, L1=L1, f1=f1, LU0=LU0, LU1=LU1, U1=U1,
               Un_bdf2=Un, fn_bdf2=fn.copy())
    # imex-lm-bdf2 coefficients (A, B, C of IMEXLM_BDF2_IntegratorAstd)
    A, B, C = [-4. / 3., 1. / 3.], [4. / 3., -2. / 3.], [2. / 3., 0., 0.]
    LM0 = rng.normal(size=npts * 5) * 1e-4
    LM1 = rng.normal(size=npts * 5) * 1e-4
    P0 = rng.normal(size=lda) * 1e-4
    P1 = rng.normal(size=lda) * 1e-4
    U2 = np.zeros(npts * 5)
    K.launch('updateMom2_LM', gm, blk, prefac, npts, dt, *A, *B, *C, LU0, LU1,
             LM0, LM1, U, U1, U2)
    M2 = M.copy()
    f2 = np.zeros(lda)
    K.launch('updateDistribution2_LM', gg, blk, prefac, lda, dt, *A, *B, *C,
             L0, L1, P0, P1, M2, f, f1, f2, U, U1, U2)
    out.update(LM0=LM0, LM1=LM1, P0=P0, P1=P1, U2_lm2=U2, f2_lm2=f2)
    # one ARS stage (q = 2, ars-222 coefficients) and the SSPL weighting
    # (q = 2, sspl-222 weights), as ARSabcIntegratorAstd / SSPLabcIntegratorAstd
    # call updateMom2_ARS, updateDistribution2_ARS, updateDistributionWeight2_SSPL
    gam = 1. - (2. ** 0.5) / 2.
    dl = 1. - 1. / (2. * gam)
    _a, a = [dl, 1 - dl], [1 - gam, gam]
    U2a = np.zeros(npts * 5)
    K.launch('updateMom2_ARS', gm, blk, prefac, npts, dt, *_a, *a, LU0, LU1,
             U, U1, U2a)
    M1 = np.zeros(lda)
    K.launch('cmaxwellian', gg, blk, lda, cx, cy, cz, M1, U1)
    M2a = np.zeros(lda)
    K.launch('cmaxwellian', gg, blk, lda, cx, cy, cz, M2a, U2a)
    f2a = np.zeros(lda)
    K.launch('updateDistribution2_ARS', gg, blk, prefac, lda, dt, *_a, *a,
             L0, L1, U, U1, U2a, M1, M2a, f, f1, f2a)
    f2s = f1 * (1 + 0.01 * rng.uniform(-1, 1, lda))
    f3 = np.zeros(lda)
    K.launch('updateDistributionWeight2_SSPL', gg, blk, prefac, lda, dt,
             0.5, 0.5, 0.5, 0.5, L0, L1, U, U1, U2a, M1, M2a, f, f1, f2s, f3)
    out.update(ars_a=np.array(_a), ars_A=np.array(a), U2_ars=U2a, M1_ars=M1,
               M2_ars=M2a, f2_ars=f2a, f2_sspl=f2s, f3_sspl=f3)
    return out


def golden_penalty_model(name, nalph, Nv=8, npts=6, omega=0.81, prefac=3.7,
                         Pr=2. / 3.):
    """The ES-BGK / Shakov penalty kernels (astd esbgk-direct-gll.mako,
    shakov-direct-gll.mako) on seeded data: moment normalisation + Gaussian,
    collide, the BDF2 and IMEX-LM2 moment and distribution updates, called
    the way the reference's integrators call them."""
    from oracle.ref_build import RefModule, grid_for, render_template
    vsize = Nv ** 3
    src = render_template(
        'dgfs1D/astd/kernels/scattering/%s.mako' % name, vsize=vsize,
        nalph=nalph, omega=omega, Pr=Pr, dtype='double', nbdf=[1, 2],
        nars=[1, 2])
    K = RefModule(src, tag=name.split('-')[0])
    rng = np.random.default_rng(SEED + 13 + nalph)
    L = 5.0
    c0 = np.linspace(-L + L / Nv, L - L / Nv, Nv)
    g = np.meshgrid(c0, c0, c0, indexing='ij')
    cv = np.stack([x.ravel() for x in g])
    cw = (2 * L / Nv) ** 3
    f = np.stack([_maxwellian_noise(cv, rng, rho=rng.uniform(0.5, 2))
                  for _ in range(npts)]).ravel()
    c2 = np.sum(cv * cv, axis=0)
    rows = [np.ones(vsize), cv[0], cv[1], cv[2], c2, cv[0] ** 2, cv[1] ** 2,
            cv[2] ** 2, cv[0] * cv[1], cv[1] * cv[2], cv[2] * cv[0],
            c2 * cv[0], c2 * cv[1], c2 * cv[2]][:nalph]
    phi = np.vstack(rows) * cw
    U = np.ascontiguousarray((f.reshape(npts, vsize) @ phi.T).ravel())
    blk = 256
    lda = npts * vsize
    gg = grid_for(lda, blk)
    gm = grid_for(npts, blk)
    cx, cy, cz = (np.ascontiguousarray(cv[i]) for i in range(3))

    def gauss(Ux):
        nU = Ux.copy()
        K.launch('momentNorm', gm, blk, npts, nU)
        Mx = np.zeros(lda)
        K.launch('cmaxwellian', gg, blk, lda, cx, cy, cz, Mx, nU)
        return Mx, nU
    M, normU = gauss(U)
    Q = np.zeros(lda)
    K.launch('collide', gg, blk, prefac, lda, M, U, f, Q)
    out = dict(Nv=Nv, npts=npts, omega=omega, prefac=prefac, Pr=Pr,
               nalph=nalph, cv=cv, cw=cw, f=f, U=U, normU=normU, M=M, Q=Q)
    dt = 0.01
    L0 = rng.normal(size=lda) * 1e-3
    L1 = rng.normal(size=lda) * 1e-3
    f1 = f * (1 + 0.01 * rng.uniform(-1, 1, lda))
    LU0 = rng.normal(size=npts * nalph) * 1e-3
    LU1 = rng.normal(size=npts * nalph) * 1e-3
    U1 = U * (1 + 0.01 * rng.uniform(-1, 1, U.shape))
    Un = np.zeros(npts * nalph)
    # bdf-222 coefficients, called as Bdf222IntegratorAstd does
    a1, a2, a3, g1, g2, b = 1. / 3., -4. / 3., 1., -2. / 3., 4. / 3., 2. / 3.
    K.launch('updateMom2_BDF', gm, blk, prefac, npts, dt, a1, U, -g1, LU0,
             a2, U1, -g2, LU1, a3, Un, b)
    Mn, _ = gauss(Un)
    fn = np.zeros(lda)
    K.launch('updateDistribution2_BDF', gg, blk, prefac, lda, dt, a1, f, -g1,
             L0, a2, f1, -g2, L1, b, Mn, a3, Un, fn)
    out.update(dt=dt, L0=L0, L1=L1, f1=f1, LU0=LU0, LU1=LU1, U1=U1,
               Un_bdf2=Un, Mn_bdf2=Mn, fn_bdf2=fn)
    # imex-lm-bdf2 coefficients (A, B, C of IMEXLM_BDF2_IntegratorAstd)
    A, B, C = [-4. / 3., 1. / 3.], [4. / 3., -2. / 3.], [2. / 3., 0., 0.]
    LM0 = rng.normal(size=npts * nalph) * 1e-4
    LM1 = rng.normal(size=npts * nalph) * 1e-4
    P0 = rng.normal(size=lda) * 1e-4
    P1 = rng.normal(size=lda) * 1e-4
    U2 = np.zeros(npts * nalph)
    K.launch('updateMom2_LM', gm, blk, prefac, npts, dt, *A, *B, *C, LU0, LU1,
             LM0, LM1, U, U1, U2)
    M2, _ = gauss(U2)
    f2 = np.zeros(lda)
    K.launch('updateDistribution2_LM', gg, blk, prefac, lda, dt, *A, *B, *C,
             L0, L1, P0, P1, M2, f, f1, f2, U, U1, U2)
    out.update(LM0=LM0, LM1=LM1, P0=P0, P1=P1, U2_lm2=U2, M2_lm2=M2,
               f2_lm2=f2)
    return out


def golden_limiter(R, K=3, Ne=8, Nv=4):
    """The linear slope limiter of dgfsABstd1D (``[time-integrator] limiter =
    1``): the reference basis' cell-average and linear-derivative operators
    (basis.py:289-301, captured by letting get_mm_kernel return its matrix)
    and its limitLin kernel (astd/kernels/limiters.mako:17-76) on a seeded
    step profile."""
    from oracle.ref_build import RefModule, grid_for, render_template
    ini = STD_INI.format(basis='nodal-sem-gll', Nv=Nv, Nrho=2, M=6, dev=5.0)
    ini = ini.replace('Ne = 4', 'Ne = %d' % Ne).replace('K = 3', 'K = %d' % K)
    cfg = R.Dictionary(ini)
    old = R.basis.get_mm_kernel
    R.basis.get_mm_kernel = lambda m, *a, **k: np.array(m, dtype=float)
    try:
        b = R.basis.NodalSemGLL(cfg)
    finally:
        R.basis.get_mm_kernel = old
    # the gimmik kernels drop entries below 1e-15 (util.py:16-26)
    import dgfs1D.util as rutil
    Aavg = rutil.filter_tol(b.computeCellAvgKern.copy())
    Adr = rutil.filter_tol(b.extractDrLinKern.copy())
    xlo, xhi = 0.0, 1.0   # nondimensional mesh (xhi - xlo = H0)
    x = np.linspace(xlo, xhi, Ne + 1)
    jac = 0.5 * np.diff(x)
    invjac = (1.0 / jac).reshape(Ne, 1)
    xsol = np.array([0.5 * (x[j] + x[j + 1]) + jac[j] * b.z for j in range(Ne)]).T
    vsize = Nv ** 3
    rng = np.random.default_rng(SEED + 29)
    prof = 1.0 + 0.5 * np.tanh((xsol - 0.5) / 0.05)
    amp = rng.uniform(0.5, 1.5, vsize)
    u = (prof[:, :, None] * amp[None, None, :]
         * (1 + 0.05 * rng.uniform(-1, 1, (K, Ne, vsize)))).ravel()
    U = u.reshape(K, Ne, vsize)
    uavg = np.einsum('kj,jev->kev', Aavg, U).ravel()
    ulx = (np.einsum('kj,jev->kev', Adr, U) * invjac[None, :, 0, None]).ravel()
    src = render_template('dgfs1D/astd/kernels/limiters.mako', K=K, Ne=Ne,
                          vsize=vsize, nalph=5, dtype='double', invjac=invjac,
                          xsol=xsol, Dr=b.derivMat)
    Km = RefModule(src, tag='limiters')
    ulim = np.zeros(K * Ne * vsize)
    Km.launch('limitLin', grid_for(vsize, 128), 128, u, ulx, uavg, ulim)
    return dict(K=K, Ne=Ne, Nv=Nv, z=b.z, Aavg=Aavg, Adr=Adr,
                derivMat=b.derivMat, invjac=invjac.ravel(), xsol=xsol, u=u,
                uavg=uavg, ulx=ulx, ulim=ulim)


def golden_upwind(R, Nv=8, Ne=5, K=3):
    """The explicit right-hand side of dgfsABUstd1D (abstdu.py:295-383): the
    reference basis' upwind operators Dp, Dm (basis.py:304-312, captured by
    letting get_mm_kernel return its matrix), its std.mako and upwind.mako
    kernels and boundary kernels, composed as explicit() composes them; two
    boundary set-ups (one-rank dgfs-cyclic on both ends, whose traces are
    swapped, and dgfs-inlet-nondim / dgfs-vanish); and the positivity limiter
    limitPos of limiters.mako on data with negative values."""
    from oracle.ref_build import RefModule, grid_for, render_template
    import dgfs1D.util as util
    ini = STD_INI.format(basis='nodal-sem-gll', Nv=Nv, Nrho=2, M=6, dev=5.0)
    ini = ini.replace('Ne = 4', 'Ne = %d' % Ne).replace('K = 3', 'K = %d' % K)
    cfg = R.Dictionary(ini)
    vm = R.vstd.DGFSVelocityMeshStd(cfg)
    old = R.basis.get_mm_kernel
    R.basis.get_mm_kernel = lambda m, *a, **k: np.array(m, dtype=float)
    try:
        b = R.basis.NodalSemGLL(cfg)
    finally:
        R.basis.get_mm_kernel = old
    Dp, Dm = np.array(b.DpKern), np.array(b.DmKern)
    Nqf, vsize = b.Nqf, vm.vsize()
    xmesh = np.linspace(0., 1., Ne + 1)
    h = np.diff(xmesh).reshape(-1, 1)
    jac, invjac = h / 2., 2. / h
    mapL, mapR = np.arange(Ne + 1) + (Nqf - 1) * Ne - 1, np.arange(Ne + 1)
    mapL[0], mapR[-1] = 0, Ne * Nqf - 1
    xsol = np.array([0.5 * (xmesh[j] + xmesh[j + 1]) + jac[j] * b.z
                     for j in range(Ne)]).T
    args = dict(K=K, Ne=Ne, Nq=K, vsize=vsize, dtype='double', mapL=mapL,
                mapR=mapR, offsetL=0, offsetR=len(mapR) - 1, invjac=invjac,
                gRD=b.gRD, gLD=b.gLD, xsol=xsol)
    SK = RefModule(render_template('dgfs1D/std/kernels/std.mako', **args), tag='std_u')
    UK = RefModule(render_template('dgfs1D/astd/kernels/upwind.mako', **args), tag='upwind')
    LK = RefModule(render_template('dgfs1D/astd/kernels/limiters.mako', nalph=5,
                                   Dr=b.derivMat, **args), tag='limiters_u')
    blk = 128
    gv = grid_for(vsize, blk)
    filt = util.filter_tol

    def mm(A, B):
        return np.ascontiguousarray(
            (filt(np.array(A, dtype=np.float64)) @ B.reshape(A.shape[1], -1)).ravel())

    cvx = np.ascontiguousarray(vm.cv()[0])
    rng = np.random.default_rng(SEED + 37)
    u = np.stack([_maxwellian_noise(vm.cv(), rng, rho=rng.uniform(0.5, 1.5))
                  for _ in range(K * Ne)]).reshape(K, Ne, vsize)
    u = np.ascontiguousarray(u.ravel())
    inlet = dict(rho=1.1, ux=0.2, T=0.95)
    uin = np.array([inlet['ux'], 0, 0]).reshape(3, 1)
    f_in = (inlet['rho'] / (np.pi * inlet['T']) ** 1.5) * np.exp(
        -np.sum((vm.cv() - uin) ** 2, axis=0) / inlet['T'])
    bmods = {}
    for kind, nl in (('dgfs-cyclic', -1.), ('dgfs-cyclic', 1.),
                     ('dgfs-inlet-nondim', -1.), ('dgfs-vanish', 1.)):
        src = render_template('dgfs1D/std/kernels/bcs/%s.mako' % kind, dtype='double',
                              vsize=vsize, cw=vm.cw(), nl=nl, x=0.0, u=inlet['ux'])
        bmods[kind, nl] = RefModule(src, tag='%s%d' % (kind.replace('-', '_'), nl > 0))
    out = {}
    for case, (kl, kr) in (('cyclic', ('dgfs-cyclic', 'dgfs-cyclic')),
                           ('inlet_vanish', ('dgfs-inlet-nondim', 'dgfs-vanish'))):
        usolF = mm(b._Bqf.T, u)
        uL, uR = np.zeros((Ne + 1) * vsize), np.zeros((Ne + 1) * vsize)
        SK.launch('extract_left', gv, blk, usolF, uL)
        SK.launch('extract_right', gv, blk, usolF, uR)
        bcL, bcR, bcT = np.zeros(vsize), np.zeros(vsize), np.zeros(vsize)
        SK.launch('transfer_bc_left', gv, blk, uL, bcL)
        SK.launch('transfer_bc_right', gv, blk, uR, bcR)
        if kr == 'dgfs-cyclic':          # abstdu.py:330-331 on one rank
            bcT[:] = bcL
            bcL[:] = bcR
            bcR[:] = bcT
        for kind, nl, bcv, ins in ((kl, -1., bcL, 'insert_bc_left'),
                                   (kr, 1., bcR, 'insert_bc_right')):
            BK = bmods[kind, nl]
            if kind == 'dgfs-cyclic':
                BK.launch('applyBC', gv, blk, bcv, bcT, cvx)
            elif kind == 'dgfs-inlet-nondim':
                BK.launch('applyBC', gv, blk, bcv, bcT, cvx, f_in, 0.0)
            else:
                BK.launch('applyBC', gv, blk, bcv, bcT, cvx, 0.0)
            SK.launch(ins, gv, blk, bcT, uL if nl < 0 else uR)
        jL, jR = np.zeros_like(uL), np.zeros_like(uR)
        UK.launch('uflux', gv, blk, uL, uR, cvx, jL, jR)
        f, g = np.zeros_like(u), np.zeros_like(u)
        UK.launch('splitFlux', grid_for(K * Ne * vsize, blk), blk, cvx, u, f, g)
        ux = mm(Dm, f)
        f = mm(Dp, g)
        ux = -(ux + f)
        SK.launch('totalFlux', gv, blk, ux, cvx, jL, jR)
        SK.launch('mul_by_invjac', gv, blk, ux)
        out['rhs_' + case] = mm(b._B.T, ux)
    # positivity limiter on data with negative values
    w = u.copy().reshape(K, Ne, vsize)
    w[0, :, ::7] -= 0.02
    w[-1, :, 3::11] -= 0.05
    w = np.ascontiguousarray(w.ravel())
    uavg = mm(b.computeCellAvgKern, w)
    ulim = np.zeros_like(w)
    LK.launch('limitPos', gv, blk, w.copy(), uavg, ulim)
    out.update(u=u, K=K, Ne=Ne, Nv=Nv, Dp=Dp, Dm=Dm, cv=vm.cv(), cw=vm.cw(),
               invjac=invjac.ravel(), inlet=np.array([inlet['rho'], inlet['ux'],
                                                     inlet['T']]),
               wpos=w, wpos_lim=ulim)
    return out


def golden_entropy(R, Nv=8, Ne=4, K=3):
    """The explicit right-hand side of dgfsABE2std1D (abstde2.py:340-380):
    the entropy-stable volume term eDeriv of limiters.mako (logarithmic mean)
    with the std.mako fluxes, lifting and invjac, and diffuse walls, composed
    as explicit() composes them, on data whose nodal values differ enough to
    take both branches of the logarithmic mean."""
    from oracle.ref_build import RefModule, grid_for, render_template
    import dgfs1D.util as util
    ini = STD_INI.format(basis='nodal-sem-gll', Nv=Nv, Nrho=2, M=6, dev=5.0)
    ini = ini.replace('Ne = 4', 'Ne = %d' % Ne).replace('K = 3', 'K = %d' % K)
    cfg = R.Dictionary(ini)
    vm = R.vstd.DGFSVelocityMeshStd(cfg)
    b = R.basis.NodalSemGLL(cfg)
    Nqf, vsize = b.Nqf, vm.vsize()
    xmesh = np.linspace(0., 1., Ne + 1)
    h = np.diff(xmesh).reshape(-1, 1)
    jac, invjac = h / 2., 2. / h
    mapL, mapR = np.arange(Ne + 1) + (Nqf - 1) * Ne - 1, np.arange(Ne + 1)
    mapL[0], mapR[-1] = 0, Ne * Nqf - 1
    xsol = np.array([0.5 * (xmesh[j] + xmesh[j + 1]) + jac[j] * b.z
                     for j in range(Ne)]).T
    args = dict(K=K, Ne=Ne, Nq=K, vsize=vsize, dtype='double', mapL=mapL,
                mapR=mapR, offsetL=0, offsetR=len(mapR) - 1, invjac=invjac,
                gRD=b.gRD, gLD=b.gLD, xsol=xsol)
    SK = RefModule(render_template('dgfs1D/std/kernels/std.mako', **args), tag='std_e')
    LK = RefModule(render_template('dgfs1D/astd/kernels/limiters.mako', nalph=5,
                                   Dr=b.derivMat, **args), tag='limiters_e')
    blk = 128
    gv = grid_for(vsize, blk)
    filt = util.filter_tol

    def mm(A, B):
        return np.ascontiguousarray(
            (filt(np.array(A, dtype=np.float64)) @ B.reshape(A.shape[1], -1)).ravel())

    cvx = np.ascontiguousarray(vm.cv()[0])
    rng = np.random.default_rng(SEED + 41)
    u = np.stack([_maxwellian_noise(vm.cv(), rng, rho=rng.uniform(0.3, 2.0))
                  for _ in range(K * Ne)]).reshape(K, Ne, vsize)
    u = np.ascontiguousarray(u.ravel())
    walls = {}
    for side, nl, uy in (('L', -1., -0.1), ('R', 1., 0.1)):
        u_w = np.array([0., uy, 0.]).reshape(3, 1)
        f0 = (1.0 / np.pi ** 1.5) * np.exp(-np.sum((vm.cv() - u_w) ** 2, axis=0))
        bsrc = render_template('dgfs1D/std/kernels/bcs/dgfs-wall-diffuse.mako',
                               dtype='double', vsize=vsize, cw=vm.cw(), ux=0.0,
                               nl=nl, x=0.0)
        walls[side] = (RefModule(bsrc, tag='wall_e' + side), f0)
    usolF = mm(b._Bqf.T, u)
    uL, uR = np.zeros((Ne + 1) * vsize), np.zeros((Ne + 1) * vsize)
    SK.launch('extract_left', gv, blk, usolF, uL)
    SK.launch('extract_right', gv, blk, usolF, uR)
    bcL, bcR, bcT = np.zeros(vsize), np.zeros(vsize), np.zeros(vsize)
    SK.launch('transfer_bc_left', gv, blk, uL, bcL)
    SK.launch('transfer_bc_right', gv, blk, uR, bcR)
    for side, bcv, ins in (('L', bcL, 'insert_bc_left'), ('R', bcR, 'insert_bc_right')):
        BK, f0 = walls[side]
        num, den = np.zeros(vsize), np.zeros(vsize)
        BK.launch('updateBC', gv, blk, bcv, cvx, f0, num, den, 0.0)
        nden = np.array([-(np.sum(num) / np.sum(den))])
        BK.launch('applyBC', gv, blk, bcv, bcT, cvx, f0, nden, 0.0)
        SK.launch(ins, gv, blk, bcT, uL if side == 'L' else uR)
    jL, jR = np.zeros_like(uL), np.zeros_like(uR)
    SK.launch('flux', gv, blk, uL, uR, cvx, jL, jR)
    ux = np.zeros_like(u)
    LK.launch('eDeriv', gv, blk, cvx, u, ux)
    SK.launch('totalFlux', gv, blk, ux, cvx, jL, jR)
    SK.launch('mul_by_invjac', gv, blk, ux)
    rhs = mm(b._B.T, ux)
    return dict(u=u, rhs=rhs, K=K, Ne=Ne, Nv=Nv, cv=vm.cv(), cw=vm.cw(),
                invjac=invjac.ravel(), derivMat=b.derivMat,
                f0L=walls['L'][1], f0R=walls['R'][1])


def golden_std_relax(R, Nv=8, omega=0.81, prefac=3.7, Pr=2. / 3.):
    """The explicit relaxation fs of dgfsStd1D's bgk-, shakov- and
    esbgk-direct-gll (std/scattering.py:1320-1371, 1764-1846, 1540-1637): the
    kernels of std/kernels/scattering/*-direct-gll.mako driven in fs's order
    on one point, with NumPy sums in place of the block reductions of sum_."""
    from oracle.ref_build import RefModule, grid_for, render_template
    vsize = Nv ** 3
    L = 5.0
    c0 = np.linspace(-L + L / Nv, L - L / Nv, Nv)
    g = np.meshgrid(c0, c0, c0, indexing='ij')
    cv = np.stack([x.ravel() for x in g])
    cw = (2 * L / Nv) ** 3
    cx, cy, cz = (np.ascontiguousarray(cv[i]) for i in range(3))
    rng = np.random.default_rng(SEED + 43)
    u = np.array([0.1, -0.05, 0.02]).reshape(3, 1)
    f = 1.1 / (np.pi * 0.9) ** 1.5 * np.exp(-np.sum((cv - u) ** 2, axis=0) / 0.9)
    f = np.ascontiguousarray(f * (1 + 0.05 * rng.uniform(-1, 1, vsize)))
    blk = 128
    gv = grid_for(vsize, blk)
    one = lambda v: np.array([float(v)])
    out = dict(f=f, cv=cv, cw=cw, omega=omega, prefac=prefac, Pr=Pr, Nv=Nv)
    for name in ('bgk', 'shakov', 'esbgk'):
        src = render_template('dgfs1D/std/kernels/scattering/%s-direct-gll.mako' % name,
                              cw=cw, vsize=vsize, prefac=prefac, nalph=5,
                              nalphSk=8, nalphES=10, omega=omega, Pr=Pr, block_size=256,
                              Ne=1, dtype='double')
        K = RefModule(src, tag='std_%s_direct' % name)
        floc = np.zeros(vsize)
        K.launch('flocKern', gv, blk, 0, 0, f, floc)
        m10, m11, m12 = np.zeros(vsize), np.zeros(vsize), np.zeros(vsize)
        K.launch('mom1', gv, blk, cx, cy, cz, floc, m10, m11, m12)
        moms = [one(np.sum(floc)), one(np.sum(m10)), one(np.sum(m11)),
                one(np.sum(m12))]
        K.launch('mom01Norm', 1, 1, *moms)
        Q = np.zeros(vsize)
        if name == 'bgk':
            m2 = np.zeros(vsize)
            K.launch('mom2', gv, blk, cx, cy, cz, floc, m2, *moms)
            moms.append(one(np.sum(m2)))
            K.launch('equiDistInit', 1, 1, *moms)
            fe = np.zeros(vsize)
            K.launch('output', gv, blk, 0, 0, 0, *moms, fe, floc, Q, cx, cy, cz)
        elif name == 'esbgk':
            m2 = np.zeros(vsize)
            K.launch('mom2', gv, blk, cx, cy, cz, floc, m2, *moms)
            moms.append(one(np.sum(m2)))
            K.launch('equiDistInit', 1, 1, *moms)
            fe = np.zeros(vsize)
            K.launch('equiDistCompute', gv, blk, cx, cy, cz, fe, *moms)
            es = [np.zeros(vsize) for _ in range(6)]
            K.launch('mom2ES', gv, blk, cx, cy, cz, floc, fe, *moms[:4], *es)
            momsES = [one(0.0) for _ in range(4)] + [one(np.sum(x)) for x in es]
            K.launch('mom2ESNorm', 1, 1, *moms, *momsES)
            feES = np.zeros(vsize)
            K.launch('equiESDistCompute', gv, blk, cx, cy, cz, feES, *momsES)
            K.launch('output', gv, blk, 0, 0, 0, moms[0], moms[4], feES, floc, Q)
        else:
            m2, q1, q2, q3 = (np.zeros(vsize) for _ in range(4))
            K.launch('mom23Sk', gv, blk, cx, cy, cz, floc, *moms, m2, q1, q2, q3)
            sk = moms + [one(np.sum(x)) for x in (m2, q1, q2, q3)]
            K.launch('mom23SkNorm', 1, 1, *sk)
            feSk = np.zeros(vsize)
            K.launch('equiSkDistCompute', gv, blk, cx, cy, cz, feSk, *sk)
            K.launch('output', gv, blk, 0, 0, 0, sk[0], sk[4], feSk, floc, Q)
        out['Q_' + name] = Q
    return out


def golden_moments(R, Nv=8, Ne=4, K=3):
    """Bulk moments of the reference's writers: DGFSMomWriterStd and
    DGFSMomWriterBi ``_compute_moments_1D`` (std/moments.py:11-70,
    bi/moments.py:11-113) on seeded drifting Maxwellians, including a mixture
    whose second species is absent (the below-1e-10 branch)."""
    import warnings
    from dgfs1D.std.moments import DGFSMomWriterStd
    from dgfs1D.bi.moments import DGFSMomWriterBi
    rng = np.random.default_rng(SEED + 31)
    out = {}

    class _Dev:               # what .get() returns, as a GPUArray would
        def __init__(self, a):
            self.a = a

        def get(self):
            return self.a

    def drift(cv, rho, ux, uy, T, mass=1.0):
        c2 = ((cv[0] - ux) ** 2 + (cv[1] - uy) ** 2 + cv[2] ** 2)
        return rho * (mass / (np.pi * T)) ** 1.5 * np.exp(-mass * c2 / T)

    def field(cv, K, Ne, mass, rho, T):
        f = np.empty((K, Ne, cv.shape[1]))
        for k in range(K):
            for e in range(Ne):
                f[k, e] = drift(cv, rho * rng.uniform(0.8, 1.2),
                                rng.uniform(-0.3, 0.3), rng.uniform(-0.3, 0.3),
                                T * rng.uniform(0.8, 1.2), mass)
        return f * (1 + 0.02 * rng.uniform(-1, 1, f.shape))

    cfg = R.Dictionary(STD_INI.format(basis='nodal-sem-gll', Nv=Nv, Nrho=2,
                                      M=6, dev=5.0).replace('Ne = 4', 'Ne = %d' % Ne))
    old = R.basis.get_mm_kernel
    R.basis.get_mm_kernel = lambda m, *a, **k: None
    try:
        b = R.basis.NodalSemGLL(cfg)
    finally:
        R.basis.get_mm_kernel = old
    vm = R.vstd.DGFSVelocityMeshStd(cfg)
    f = field(vm.cv(), K, Ne, 1.0, 1.0, 1.0)
    w = object.__new__(DGFSMomWriterStd)
    w.vm, w.im = vm, b.interpMat
    w._bulksoln = np.zeros((b.interpMat.shape[1], Ne, 10))
    w._compute_moments_1D(_Dev(f.ravel()))
    out.update(std_f=f, std_mom=w._bulksoln.copy(), std_cw=vm.cw(),
               std_cv=vm.cv(), std_T0=vm.T0(), std_rho0=vm.rho0(),
               std_u0=vm.u0(), std_molarMass0=vm.molarMass0(),
               interpMat=b.interpMat)
    cfg = R.Dictionary(BI_INI.format(Nv=Nv, Nrho=2, M=6, Mpre=12, dev=5.0)
                       .replace('Ne = 2', 'Ne = %d' % Ne))
    vm = R.vbi.DGFSVelocityMeshBi(cfg)
    ms = vm.masses()
    for tag, absent in (('mix', False), ('absent', True)):
        fs = [field(vm.cv(), K, Ne, ms[0], 0.5, 1.0),
              field(vm.cv(), K, Ne, ms[1], 0.5, 1.2)]
        if absent:
            fs[1][:] = 0.0
        w = object.__new__(DGFSMomWriterBi)
        w.vm, w.im = vm, b.interpMat
        Nqr = b.interpMat.shape[1]
        w._bulksoln = np.zeros((Nqr, Ne, 7 * 2))
        w._bulksolntot = np.zeros((Nqr, Ne, 4))
        with warnings.catch_warnings():
            warnings.simplefilter('ignore')
            w._compute_moments_1D([_Dev(x.ravel()) for x in fs])
        out['bi_%s_f0' % tag], out['bi_%s_f1' % tag] = fs
        out['bi_%s_mom' % tag] = w._bulksoln.copy()
    out.update(bi_cw=vm.cw(), bi_cv=vm.cv(), bi_masses=np.array(ms),
               bi_T0=vm.T0(), bi_rho0=vm.rho0(), bi_u0=vm.u0(),
               bi_molarMass0=vm.molarMass0(), bi_R0=vm.R0, bi_NA=vm.NA)
    return out


def golden_setup(R):
    """Velocity meshes, rules and DG bases from the reference setup code."""
    out = {}
    for Nv, Nrho, M, dev in [(16, 8, 6, 5.0), (32, 16, 16, 6.0),
                             (24, 12, 6, 5.0)]:
        cfg = R.Dictionary(STD_INI.format(basis='nodal-sem-gll', Nv=Nv,
                                          Nrho=Nrho, M=M, dev=dev))
        vm = R.vstd.DGFSVelocityMeshStd(cfg)
        sm = object.__new__(R.VHSGLL)
        sm.cfg, sm.vm = cfg, vm
        sm.load_parameters()
        key = f'std_N{Nv}_M{M}_R{Nrho}'
        out[key + '_L'] = vm.L()
        out[key + '_qz'] = vm.qz()
        out[key + '_qw'] = vm.qw()
        out[key + '_sz'] = vm.sz()
        out[key + '_sw'] = vm.sw()
        out[key + '_cw'] = vm.cw()
        out[key + '_c0'] = vm.cv()[2, :Nv]
        out[key + '_prefac'] = sm._prefactor
    for kind in ('nodal-sem-gll', 'nodal-gll'):
        cfg = R.Dictionary(STD_INI.format(basis=kind, Nv=8, Nrho=4, M=6,
                                          dev=5.0))
        cls = {'nodal-sem-gll': R.basis.NodalSemGLL,
               'nodal-gll': R.basis.NodalGLL}[kind]
        b = cls(cfg)
        key = 'basis_' + kind.replace('-', '_')
        out[key + '_z'] = b.z
        out[key + '_gLD'] = np.asarray(b.gLD)
        out[key + '_gRD'] = np.asarray(b.gRD)
        out[key + '_derivMat'] = b.derivMat
        out[key + '_interpMat'] = b.interpMat
        out[key + '_U'] = np.stack(b._U)
        out[key + '_V'] = np.stack(b._V)
        out[key + '_sigModes'] = np.array([list(s) for s in b.sigModes])
        out[key + '_Bqf'] = b._Bqf
    for n in (2, 3, 4, 6, 8, 12, 16, 24):
        z, w = R.quadratures.zwgj(n, 0., 0.)
        out[f'zwgj_{n}_z'], out[f'zwgj_{n}_w'] = z, w
        z, w = R.quadratures.zwglj(n, 0., 0.)
        out[f'zwglj_{n}_z'], out[f'zwglj_{n}_w'] = z, w
    return out


def main():
    R = _import_reference()
    np.savez_compressed(os.path.join(HERE, 'setup.npz'), **golden_setup(R))
    np.savez_compressed(os.path.join(HERE, 'vhs_N8.npz'), **golden_vhs(R))
    np.savez_compressed(os.path.join(HERE, 'vss_N8.npz'), **golden_vss(R))
    for kind in ('nodal-sem-gll', 'nodal-gll'):
        np.savez_compressed(
            os.path.join(HERE, 'dg_%s_N8.npz' % kind.replace('-', '_')),
            **golden_dg(R, kind))
    np.savez_compressed(os.path.join(HERE, 'penalty_N8.npz'),
                        **golden_penalty(R))
    penalty_models()
    np.savez_compressed(os.path.join(HERE, 'limiter_N4.npz'), **golden_limiter(R))
    np.savez_compressed(os.path.join(HERE, 'moments_N8.npz'), **golden_moments(R))
    np.savez_compressed(os.path.join(HERE, 'upwind_N8.npz'), **golden_upwind(R))
    np.savez_compressed(os.path.join(HERE, 'entropy_N8.npz'), **golden_entropy(R))
    np.savez_compressed(os.path.join(HERE, 'std_relax_N8.npz'), **golden_std_relax(R))
    for fn in sorted(os.listdir(HERE)):
        if fn.endswith('.npz'):
            print(fn, os.path.getsize(os.path.join(HERE, fn)), 'bytes')


def limiter():
    R = _import_reference()
    np.savez_compressed(os.path.join(HERE, 'limiter_N4.npz'), **golden_limiter(R))


def penalty():
    R = _import_reference()
    np.savez_compressed(os.path.join(HERE, 'penalty_N8.npz'), **golden_penalty(R))


def std_relax():
    R = _import_reference()
    np.savez_compressed(os.path.join(HERE, 'std_relax_N8.npz'), **golden_std_relax(R))


def upwind():
    R = _import_reference()
    np.savez_compressed(os.path.join(HERE, 'upwind_N8.npz'), **golden_upwind(R))


def entropy():
    R = _import_reference()
    np.savez_compressed(os.path.join(HERE, 'entropy_N8.npz'), **golden_entropy(R))


def moments():
    R = _import_reference()
    np.savez_compressed(os.path.join(HERE, 'moments_N8.npz'), **golden_moments(R))


def penalty_models():
    for name, nalph, tag in (('esbgk-direct-gll', 11, 'esbgk'),
                             ('shakov-direct-gll', 14, 'shakov')):
        np.savez_compressed(os.path.join(HERE, 'penalty_%s_N8.npz' % tag),
                            **golden_penalty_model(name, nalph))


if __name__ == '__main__':
    import sys
    if sys.argv[1:] == ['penalty-models']:
        penalty_models()
    elif sys.argv[1:] == ['limiter']:
        limiter()
    elif sys.argv[1:] == ['moments']:
        moments()
    elif sys.argv[1:] == ['upwind']:
        upwind()
    elif sys.argv[1:] == ['std-relax']:
        std_relax()
    elif sys.argv[1:] == ['penalty']:
        penalty()
    elif sys.argv[1:] == ['entropy']:
        entropy()
    else:
        main()
