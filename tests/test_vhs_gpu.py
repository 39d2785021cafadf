"""Parity of the CUDA VHS collision operator with the CPU oracle."""
import numpy as np
import pytest
import torch

from oracle.collision import vhs_gll_fs
from tests._cases import op_kwargs, vhs_case, vhs_tables

pytestmark = pytest.mark.gpu

# (N, M, Nrho, dev, full_sphere): small grids, the 12-point config shape
# (N=16, half sphere M=6, Nrho=8, [-5,5]^3) and the N=32 shape (full 12-point
# sphere, Nrho=16, [-6,6]^3)
CASES = [(8, 6, 4, 5., False), (16, 6, 8, 5., False), (32, 12, 16, 6., True)]

FP64_TOL = 1e-11   # relative L2, plain FP64 mode
FP32_TOL = 1e-5    # relative L2, FP32 mode (Maxwellian split)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope='module')
def lib():
    from dgfs1d_gpu_b200 import build
    build.build()
    from dgfs1d_gpu_b200 import _native
    return _native.lib()


@pytest.mark.parametrize('case', CASES, ids=lambda c: f'N{c[0]}')
@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_single_eval_matches_oracle(lib, case, precision):
    from dgfs1d_gpu_b200.collision import VHSOperator
    N, M, Nrho, dev, full = case
    vm, prefac, gamma, f = vhs_case(N, M, Nrho, dev, full, nslots=1)
    tab = vhs_tables(vm, gamma)
    q_ref = vhs_gll_fs(tab, prefac, f[0])
    op = VHSOperator(**op_kwargs(vm, prefac, gamma), precision=precision,
                     max_evals=4)
    dt = torch.float64
    fd = torch.tensor(f, dtype=dt, device='cuda')
    Q = torch.zeros_like(fd)
    op.eval(fd, Q)
    torch.cuda.synchronize()
    err = _rel(Q.cpu().numpy()[0], q_ref)
    tol = FP64_TOL if precision == 'fp64' else FP32_TOL
    assert err < tol, f'{precision} N={N}: rel L2 {err:.3e}'


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_batched_slots_accumulate(lib, precision):
    """Slot mapping and += semantics over a batch larger than max_evals."""
    from dgfs1d_gpu_b200.collision import VHSOperator
    N, M, Nrho, dev, full = CASES[1]
    nslots = 7
    vm, prefac, gamma, f = vhs_case(N, M, Nrho, dev, full, nslots=nslots)
    tab = vhs_tables(vm, gamma)
    op = VHSOperator(**op_kwargs(vm, prefac, gamma), precision=precision,
                     max_evals=3)
    fd = torch.tensor(f, device='cuda')
    Q0 = torch.randn_like(fd) * 1e-3
    Q = Q0.clone()
    src = torch.tensor([6, 0, 3, 5, 1], dtype=torch.int32, device='cuda')
    dst = torch.tensor([0, 1, 2, 3, 4], dtype=torch.int32, device='cuda')
    op.eval(fd, Q, src=src, dst=dst)
    torch.cuda.synchronize()
    Qh, Q0h = Q.cpu().numpy(), Q0.cpu().numpy()
    tol = FP64_TOL if precision == 'fp64' else FP32_TOL
    for i, s in enumerate(src.tolist()):
        ref = vhs_gll_fs(tab, prefac, f[s])
        assert _rel(Qh[i] - Q0h[i], ref) < tol
    for i in (5, 6):   # untouched slots
        assert np.array_equal(Qh[i], Q0h[i])


def test_float32_arrays(lib):
    """precision=float drop-in: FP32 f and Q arrays, FP32 mode."""
    from dgfs1d_gpu_b200.collision import VHSOperator
    N, M, Nrho, dev, full = CASES[1]
    vm, prefac, gamma, f = vhs_case(N, M, Nrho, dev, full, nslots=2)
    tab = vhs_tables(vm, gamma)
    op = VHSOperator(**op_kwargs(vm, prefac, gamma), precision='fp32',
                     max_evals=2, sinc_eps=1e-15)
    fd = torch.tensor(f, dtype=torch.float32, device='cuda')
    Q = torch.zeros_like(fd)
    op.eval(fd, Q)
    torch.cuda.synchronize()
    for s in range(2):
        ref = vhs_gll_fs(tab, prefac, f[s].astype(np.float32).astype(np.float64))
        assert _rel(Q.cpu().numpy()[s].astype(np.float64), ref) < FP32_TOL


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_matches_reference_kernel_golden(lib, precision):
    """CUDA path vs the reference's own kernels (tests/golden/vhs_N8.npz)."""
    import os
    from dgfs1d_gpu_b200.collision import VHSOperator
    g = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'vhs_N8.npz'))
    N = int(g['Nv'])
    op = VHSOperator(N=N, L=float(g['L']), qz=g['qz'], qw=g['qw'], sz=g['sz'],
                     sw=float(g['sw']), sphere_factor=2.0,
                     gamma=float(g['gamma']), prefac=float(g['prefac']),
                     cw=float(g['cw']), c0=g['cv'][2, :N], precision=precision,
                     max_evals=8)
    f = torch.tensor(g['f'], device='cuda')
    Q = torch.zeros_like(f)
    op.eval(f, Q)
    torch.cuda.synchronize()
    tol = FP64_TOL if precision == 'fp64' else FP32_TOL
    ref = g['Q_vhs_gll'].reshape(-1, N ** 3)
    got = Q.cpu().numpy().reshape(-1, N ** 3)
    for s in range(ref.shape[0]):
        assert _rel(got[s], ref[s]) < tol, s


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_n24(lib, precision):
    from dgfs1d_gpu_b200.collision import VHSOperator
    vm, prefac, gamma, f = vhs_case(24, 6, 12, 5., False, nslots=2)
    tab = vhs_tables(vm, gamma)
    op = VHSOperator(**op_kwargs(vm, prefac, gamma), precision=precision,
                     max_evals=2)
    fd = torch.tensor(f, device='cuda')
    Q = torch.zeros_like(fd)
    op.eval(fd, Q)
    torch.cuda.synchronize()
    tol = FP64_TOL if precision == 'fp64' else FP32_TOL
    for s in range(2):
        assert _rel(Q.cpu().numpy()[s], vhs_gll_fs(tab, prefac, f[s])) < tol


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_conservation_projection(lib, precision):
    """After projection the five moments of Q vanish to 1e-12 (relative to
    the moments of |Q|), and the correction is the minimal-L2 one."""
    from dgfs1d_gpu_b200.collision import VHSOperator
    N, M, Nrho, dev, full = CASES[2]
    vm, prefac, gamma, f = vhs_case(N, M, Nrho, dev, full, nslots=2,
                                    noise=0.05)
    op = VHSOperator(**op_kwargs(vm, prefac, gamma), precision=precision,
                     max_evals=2)
    fd = torch.tensor(f, device='cuda')
    Q0 = torch.zeros_like(fd)
    op.eval(fd, Q0)
    op.set_projection(True)
    Q1 = torch.zeros_like(fd)
    op.eval(fd, Q1)
    torch.cuda.synchronize()
    cv, cw = vm.cv, vm.cw
    phi = np.vstack([np.ones(N ** 3), cv, np.sum(cv ** 2, axis=0)])
    G = (phi * cw) @ phi.T
    for s in range(2):
        q0, q1 = Q0.cpu().numpy()[s], Q1.cpu().numpy()[s]
        scale = np.abs(phi * cw) @ np.abs(q0)
        mom1 = (phi * cw) @ q1
        assert np.all(np.abs(mom1) <= 1e-12 * scale), mom1 / scale
        lam = np.linalg.solve(G, (phi * cw) @ q0)
        assert _rel(q1, q0 - lam @ phi) < 1e-12


@pytest.mark.parametrize('case', [(16, 6, 8, 5., False), (24, 12, 12, 5., True),
                                  (32, 12, 16, 6., True)],
                         ids=lambda c: f'N{c[0]}')
def test_fp32_cluster_variants_match_oracle(lib, case):
    """Every cluster size of the FP32 terms kernel (the autotuner's search
    space) gives the oracle's Q; the autotuner keeps one of them."""
    from dgfs1d_gpu_b200.collision import VHSOperator
    N, M, Nrho, dev, full = case
    vm, prefac, gamma, f = vhs_case(N, M, Nrho, dev, full, nslots=2)
    tab = vhs_tables(vm, gamma)
    refs = [vhs_gll_fs(tab, prefac, f[s]) for s in range(2)]
    op = VHSOperator(**op_kwargs(vm, prefac, gamma), precision='fp32',
                     max_evals=2)
    fd = torch.tensor(f, dtype=torch.float64, device='cuda')
    variants = op.variants()
    assert len(variants) >= 2
    for c in variants:
        op.set_variant(c)
        Q = torch.zeros_like(fd)
        op.eval(fd, Q)
        torch.cuda.synchronize()
        assert op.device_error() == 0, f'N={N} variant {c}: a bounded wait gave up'
        for s in range(2):
            err = _rel(Q.cpu().numpy()[s], refs[s])
            assert err < FP32_TOL, f'N={N} cluster {c}: rel L2 {err:.3e}'
    times = op.autotune(fd, torch.zeros_like(fd), reps=2)
    assert set(times) == set(variants) and op.variant in variants


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_n48_matches_oracle(lib, precision):
    """N=48 (16-CTA clusters; the FP64 terms kernel keeps its sums in global
    memory) against the oracle, hard spheres (omega = 0.5) on [-8, 8]^3, with
    a reduced sphere/radial rule so that the oracle finishes in seconds."""
    from dgfs1d_gpu_b200.collision import VHSOperator
    vm, prefac, gamma, f = vhs_case(48, 6, 4, 8.0, False, omega=0.5, nslots=2)
    tab = vhs_tables(vm, gamma)
    op = VHSOperator(**op_kwargs(vm, prefac, gamma), precision=precision,
                     max_evals=2)
    fd = torch.tensor(f, dtype=torch.float64, device='cuda')
    tol = FP64_TOL if precision == 'fp64' else FP32_TOL
    refs = [vhs_gll_fs(tab, prefac, f[s]) for s in range(2)]
    for c in (op.variants() if precision == 'fp32' else [0]):
        if c:
            op.set_variant(c)
        Q = torch.zeros_like(fd)
        op.eval(fd, Q)
        torch.cuda.synchronize()
        for s in range(2):
            err = _rel(Q.cpu().numpy()[s], refs[s])
            assert err < tol, f'N=48 {precision} variant {c} slot {s}: rel L2 {err:.3e}'



@pytest.fixture(scope='module')
def c5_case():
    """The stress configuration's rule: hard spheres (omega = 0.5), N=48 on
    [-8, 8]^3, the full 32-point spherical design, Nrho=24.  The oracle takes
    about 6 s per point on 8 host cores (2307 transforms of 48^3)."""
    vm, prefac, gamma, f = vhs_case(48, 32, 24, 8.0, True, omega=0.5, nslots=2)
    tab = vhs_tables(vm, gamma)
    refs = [vhs_gll_fs(tab, prefac, f[s]) for s in range(2)]
    return vm, prefac, gamma, f, refs


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_n48_stress_rule_matches_oracle(lib, c5_case, precision):
    """N=48 at the full stress rule (M=32 full sphere, Nrho=24): 16-CTA
    clusters with three planes per CTA in both modes, 16 merged directions."""
    from dgfs1d_gpu_b200.collision import VHSOperator
    vm, prefac, gamma, f, refs = c5_case
    op = VHSOperator(**op_kwargs(vm, prefac, gamma), precision=precision,
                     max_evals=2)
    fd = torch.tensor(f, dtype=torch.float64, device='cuda')
    Q = torch.zeros_like(fd)
    op.eval(fd, Q)
    torch.cuda.synchronize()
    tol = FP64_TOL if precision == 'fp64' else FP32_TOL
    for s in range(2):
        err = _rel(Q.cpu().numpy()[s], refs[s])
        assert err < tol, f'N=48 stress rule {precision} slot {s}: rel L2 {err:.3e}'
    op.close()


# -- bilinear Q(f, g) (``vhs``) ----------------------------------------------

def _two_inputs(vm, nslots, seed=5):
    """f: the Couette-like case distributions; g: Maxwellians of another
    temperature and bulk velocity with their own 1% noise."""
    from dgfs1d_gpu_b200.workloads import couette_distributions
    c0 = vm.cv[2, :vm.Nv]
    f = couette_distributions(c0, nslots, noise=0.01, seed=seed)
    cv = vm.cv
    rng = np.random.default_rng(seed + 1)
    u = np.array([0.05, -0.08, 0.02])[:, None]
    m = 1.1 / (np.pi * 1.2) ** 1.5 * np.exp(-np.sum((cv - u) ** 2, axis=0) / 1.2)
    g = np.stack([m * (1 + 0.01 * rng.uniform(-1, 1, m.shape))
                  for _ in range(nslots)])
    return f, g


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_bilinear_matches_reference_kernel_golden(lib, precision):
    """dgfs_vhs_eval2 vs the reference's own bilinear kernels
    (cosMul/sinMul/cplxMul/cplxMulAdd, tests/golden/vhs_N8.npz Q_vhs)."""
    import os
    from dgfs1d_gpu_b200.collision import VHSOperator
    g = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'vhs_N8.npz'))
    N = int(g['Nv'])
    op = VHSOperator(N=N, L=float(g['L']), qz=g['qz'], qw=g['qw'], sz=g['sz'],
                     sw=float(g['sw']), sphere_factor=2.0,
                     gamma=float(g['gamma']), prefac=float(g['prefac']),
                     cw=float(g['cw']), c0=g['cv'][2, :N], precision=precision,
                     max_evals=4)
    f = torch.tensor(g['f'], device='cuda').reshape(-1, N ** 3)
    gg = torch.tensor(g['g'], device='cuda').reshape(-1, N ** 3)
    Q = torch.zeros_like(f)
    op.eval2(f, gg, Q)
    torch.cuda.synchronize()
    tol = FP64_TOL if precision == 'fp64' else FP32_TOL
    ref = g['Q_vhs'].reshape(-1, N ** 3)
    got = Q.cpu().numpy()
    for s in range(ref.shape[0]):
        assert _rel(got[s], ref[s]) < tol, s


@pytest.mark.parametrize('case', [CASES[1], CASES[2]], ids=['N16', 'N32'])
@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_bilinear_matches_oracle(lib, case, precision):
    """Q(f, g) with g != f (another temperature and bulk velocity) against
    the oracle's vhs_fs, slot lists and += included."""
    from dgfs1d_gpu_b200.collision import VHSOperator
    from oracle.collision import vhs_fs
    N, M, Nrho, dev, full = case
    vm, prefac, gamma, _ = vhs_case(N, M, Nrho, dev, full, nslots=1)
    f, g = _two_inputs(vm, 3)
    tab = vhs_tables(vm, gamma)
    op = VHSOperator(**op_kwargs(vm, prefac, gamma), precision=precision,
                     max_evals=2)
    fd, gd = torch.tensor(f, device='cuda'), torch.tensor(g, device='cuda')
    Q0 = torch.randn_like(fd) * 1e-6
    Q = Q0.clone()
    src = torch.tensor([2, 0], dtype=torch.int32, device='cuda')
    dst = torch.tensor([1, 2], dtype=torch.int32, device='cuda')
    op.eval2(fd, gd, Q, src=src, dst=dst)
    torch.cuda.synchronize()
    tol = FP64_TOL if precision == 'fp64' else FP32_TOL
    got = (Q - Q0).cpu().numpy()
    for s, d in ((2, 1), (0, 2)):
        ref = vhs_fs(tab, prefac, f[s], g[s])
        assert _rel(got[d], ref) < tol, (precision, N, s)
    assert torch.equal(Q[0], Q0[0])


def test_bilinear_with_g_equal_f_is_q_ff(lib):
    """Q(f, f) through the bilinear entry equals dgfs_vhs_eval (FP64)."""
    from dgfs1d_gpu_b200.collision import VHSOperator
    N, M, Nrho, dev, full = CASES[1]
    vm, prefac, gamma, f = vhs_case(N, M, Nrho, dev, full, nslots=2)
    op = VHSOperator(**op_kwargs(vm, prefac, gamma), precision='fp64',
                     max_evals=2)
    fd = torch.tensor(f, device='cuda')
    Q1, Q2 = torch.zeros_like(fd), torch.zeros_like(fd)
    op.eval(fd, Q1)
    op.eval2(fd, fd.clone(), Q2)
    torch.cuda.synchronize()
    assert _rel(Q2.cpu().numpy(), Q1.cpu().numpy()) < 1e-12


@pytest.mark.parametrize('precision', [None, 'fp32'])
def test_vhs_plugin_fs_bilinear(lib, precision):
    """The ``vhs`` plugin's fs(d_arr_in1, d_arr_in2, d_arr_out, elem, modein,
    modeout) with two distinct arrays is Q(f, g) at slot modein*Ne + elem,
    added into slot modeout*Ne + elem (std/scattering.py:346-429); with the
    same array twice it is Q(f, f)."""
    from dgfs1d_gpu_b200.config import Config
    from dgfs1d_gpu_b200.configs import couette_std_ini
    from dgfs1d_gpu_b200.std.solver import DGFSStd1D
    from oracle.collision import VHSTables, vhs_fs, vhs_gll_fs
    ini = couette_std_ini(Nv=16, Nrho=8, M=6, precision_mode=precision)
    ini = ini.replace('type = vhs-gll', 'type = vhs')
    s = DGFSStd1D(Config(ini))
    assert s.sm.scattering_model == 'vhs'
    vm, Ne = s.vm, s.mesh.Ne
    u = s.u.reshape(-1, vm.vsize())
    g = (u * (1 + 0.05 * torch.rand_like(u))).contiguous()
    Q = torch.zeros_like(u)
    s.sm.fs(u, g, Q, 2, 1, 0)          # elem 2, modein 1, modeout 0
    s.sm.fs(u, u, Q, 3, 0, 2)          # the same array: Q(f, f)
    torch.cuda.synchronize()
    # double arrays: the sinc regulariser is the double one in both modes
    tab = VHSTables(vm.Nv(), vm.L(), vm.qz(), vm.qw(), vm.sz(), vm.sw(),
                    2 * (1 - s.sm.omega), sphere_factor=vm.sphere_factor())
    uh, gh, Qh = u.cpu().numpy(), g.cpu().numpy(), Q.cpu().numpy()
    tol = FP64_TOL if precision is None else FP32_TOL
    ref1 = vhs_fs(tab, s.sm.prefac, uh[1 * Ne + 2], gh[1 * Ne + 2])
    ref2 = vhs_gll_fs(tab, s.sm.prefac, uh[0 * Ne + 3])
    assert _rel(Qh[0 * Ne + 2], ref1) < tol
    assert _rel(Qh[2 * Ne + 3], ref2) < tol
    mask = np.ones(len(Qh), bool)
    mask[[2, 2 * Ne + 3]] = False
    assert not Qh[mask].any()
