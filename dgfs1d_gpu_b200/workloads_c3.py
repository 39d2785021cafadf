"""The uneven multi-problem batch: six single-species VHS problems with
N in {16, 24, 32, 16, 24, 32}, Ne*K spatial points in {12, 24, 40, 12, 24,
40}, M in {6, 12, 12, 6, 12, 12} (M=6: half sphere, M=12: full sphere),
Nrho = N/2, plus two binary-mixture VSS problems (N=24, Ne=6, K=3, masses
1:2, mole fractions 0.5/0.5, alpha=1.4, omega=0.81, full 12-point sphere,
Mpre=192), with seeded perturbed (bi-)Maxwellians (VSS temperatures 1 and
1.2, 2% uniform noise).  All problems run in the given precision; the VHS
problems add the FP64 conservation projection (a single VSS pair conserves
only the mass of its species, so the mixtures are not projected)."""
import math

import numpy as np
import torch

from .collision import VHSOperator, VSSOperator
from .sphericaldesign import get_sphquadrule
from .workloads import couette_distributions, vhs_mesh_params
from .quadrature import gauss_jacobi

VHS_PROBLEMS = [(16, 12, 6), (24, 24, 12), (32, 40, 12),
                (16, 12, 6), (24, 24, 12), (32, 40, 12)]


def build_c3(precision='fp32', device='cuda', seed=20261203, project=True,
             merged=False, autotune=False):
    """The eight problems as dicts (name, op, f, Q, nevals, params, fn).

    merged=True instead returns one dict per group of problems that share
    an operator -- the VHS problems of equal N (equal grids and rules here)
    and the two mixtures -- with one operator per group, ``fn`` evaluating
    every member's points in one call per kernel, and the members' dicts
    (without ops) under ``members``.  ``autotune`` (merged only) lets the
    project's autotuner pick each VHS group's terms-kernel variant (tile
    shape, radix split, staging) on the group's own merged call; the
    timings and the choice are under ``variant_ms`` and ``variant``."""
    if merged:
        if precision != 'fp32':
            raise ValueError('merged groups need the FP32 mode (the VSS array '
                             'lists are FP32 only)')
        return _build_merged(precision, device, seed, project, autotune)
    problems = []
    for i, (N, pts, M) in enumerate(VHS_PROBLEMS):
        full = M == 12
        prm = vhs_mesh_params(N, M, N // 2, 5.0 if N < 32 else 6.0, full)
        f = torch.tensor(couette_distributions(prm['c0'], pts, noise=0.02,
                                               seed=seed + i),
                         dtype=torch.float64, device=device)
        Q = torch.zeros_like(f)
        op = VHSOperator(**prm, precision=precision, max_evals=pts)
        if project:
            op.set_projection(True)
        def fn(op=op, f=f, Q=Q):
            Q.zero_()
            op.eval(f, Q)
        problems.append(dict(name=f'vhs{i}-N{N}-{pts}pts', op=op, f=f, Q=Q,
                             nevals=pts, params=prm, fn=fn))
    # two VSS mixtures, N=24, 18 points, 4 pairs each
    N, pts, M, Mpre = 24, 18, 12, 192
    masses = [1.0, 2.0]
    mr = max(masses)
    L = 5.0
    S = min(L * 2.0 / (max(4. * mr / (1. + mr), 2.) + math.sqrt(1. + mr) + 1.),
            L * 2.0 / (max(4. / (1. + mr), 2.) + math.sqrt(1. + 1.0 / mr) + 1.0))
    z, w = gauss_jacobi(N // 2)
    qz, qw = S * (1 + z), S * w
    sz = get_sphquadrule('symmetric', 'womersley', npts=M).pts
    szpre = get_sphquadrule('symmetric', 'womersley', npts=Mpre).pts
    c0 = np.linspace(-L + L / N, L - L / N, N)
    g = np.meshgrid(c0, c0, c0, indexing='ij')
    cv = np.stack([x.ravel() for x in g])
    for j in range(2):
        rng = np.random.default_rng(seed + 100 + j)
        fs = []
        for sp, T in ((0, 1.0), (1, 1.2)):
            m = 0.5 * np.exp(-masses[sp] * np.sum(cv ** 2, axis=0) / T) \
                * (masses[sp] / (np.pi * T)) ** 1.5
            fs.append(np.stack([m * (1 + 0.02 * rng.uniform(-1, 1, m.shape))
                                for _ in range(pts)]))
        omega, alpha = 0.81, 1.4
        gam = np.full((2, 2), 2 * (1 - omega))
        eta = np.full((2, 2), alpha - 1)
        pre = np.full((2, 2), 0.1)
        op = VSSOperator(N, L, qz, qw, sz, 4 * np.pi / M, szpre, masses, gam,
                         eta, pre, max_evals=pts, precision=precision)
        fd = [torch.tensor(x, device=device) for x in fs]
        Qd = [torch.zeros_like(x) for x in fd]

        def fn(op=op, fd=fd, Qd=Qd):
            for x in Qd:
                x.zero_()
            for p in range(2):
                op.eval_species(p, fd, Qd[p])
        problems.append(dict(name=f'vss{j}-N{N}-{pts}pts', op=op, f=fd, Q=Qd,
                             nevals=4 * pts, fn=fn,
                             params=dict(N=N, L=L, qz=qz, qw=qw, sz=sz,
                                         sw=4 * np.pi / M, szpre=szpre,
                                         masses=masses, gamma=gam, eta=eta,
                                         prefac=pre)))
    return problems


def _build_merged(precision, device, seed, project, autotune=False):
    from .batch import merged_vhs, merged_vss
    single = build_c3(precision, device, seed, project)
    groups = []
    vhs = [p for p in single if p['name'].startswith('vhs')]
    for N in sorted({p['params']['N'] for p in vhs}):
        members = [p for p in vhs if p['params']['N'] == N]
        prm = members[0]['params']
        tot = sum(p['nevals'] for p in members)
        op = VHSOperator(**prm, precision=precision, max_evals=tot)
        if project:
            op.set_projection(True)
        call = merged_vhs(op, [(p['f'], p['Q']) for p in members])

        def fn(call=call, members=members):
            for p in members:
                p['Q'].zero_()
            call()
        g = dict(name=f'vhs-N{N}-x{len(members)}', op=op, fn=fn,
                 nevals=tot, members=members)
        if autotune:
            g['variant_ms'] = op.autotune(call=fn)
            g['variant'] = op.variant
        groups.append(g)
    vss = [p for p in single if p['name'].startswith('vss')]
    prm = vss[0]['params']
    tot = sum(p['nevals'] // 4 for p in vss)
    op = VSSOperator(prm['N'], prm['L'], prm['qz'], prm['qw'], prm['sz'],
                     prm['sw'], prm['szpre'], prm['masses'], prm['gamma'],
                     prm['eta'], prm['prefac'], max_evals=tot,
                     precision=precision)
    call = merged_vss(op, [(p['f'], p['Q']) for p in vss])

    def fn(call=call, members=vss):
        for p in members:
            for x in p['Q']:
                x.zero_()
        call()
    groups.append(dict(name=f'vss-N{prm["N"]}-x{len(vss)}', op=op, fn=fn,
                       nevals=4 * tot, members=vss))
    for p in single:          # the members' own operators are not needed
        p['op'].close()
        p.pop('op')
        p.pop('fn')
    return groups


if __name__ == '__main__':
    # python -m dgfs1d_gpu_b200.workloads_c3 [vhs|vss|all] [stages]: run the
    # stage of the chosen problems (FP32, one call per problem) a few times
    import sys
    which = sys.argv[1] if len(sys.argv) > 1 else 'all'
    stages = int(sys.argv[2]) if len(sys.argv) > 2 else 3
    probs = [p for p in build_c3(precision='fp32')
             if which == 'all' or p['name'].startswith(which)]
    for _ in range(stages):
        for p in probs:
            p['fn']()
    torch.cuda.synchronize()
    print('ran', stages, 'stages of', [p['name'] for p in probs])
