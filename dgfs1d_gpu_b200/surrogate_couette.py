"""Surrogate-assisted steady Couette flow against the plain solver.

The learned-part experiment: Couette flow between diffuse walls at
u_y = -/+0.1 (Kn = 0.1, VHS omega = 0.81), N = 32^3 velocity grid on
[-6, 6]^3 (12-point full-sphere design, 16 radial points), Ne = 8, K = 3,
advanced with BDF2 IMEX (``imex-lm-bdf2``: Boltzmann-BGK penalty implicit,
Q - P explicit) from rest to a steady state at a 1e-8 relative change of the
bulk moments per step.

1. The plain solver (FP64 fast-spectral operator) runs to steady state: the
   reference wall time and shear stress P_xy / heat flux Q_x profiles.
2. Training pairs: seeded perturbed Maxwellians (density [0.5, 2],
   temperature [0.7, 1.5], bulk velocity [-0.3, 0.3]^3, 5% noise) and states
   harvested along a plain run, each with Q from the plain operator.
3. The FNO surrogate is trained on the GPU with the library's kernels (half
   of every batch drawn from the harvested states).
4. The solver with the fused FP32 operator (no surrogate).
5. The surrogate-assisted solver (plain operator every k = 10 calls, fallback
   above a 1e-3 residual) runs to steady state, in three modes: the surrogate
   alone between checks, the surrogate plus the defect measured at the last
   check, and the latter with the fused FP32 operator as the plain operator
   (checks and fallback).

``python -m dgfs1d_gpu_b200.surrogate_couette [--quick]`` prints one JSON
report (``--quick``: N = 16 and short budgets, for tests).
"""
import argparse
import json
import time

import numpy as np
import torch

from .astd.solver import DGFSABstd1D
from .config import Config
from .configs import couette_astd_ini
from .surrogate import FNOSurrogate
from . import surrogate_train as st


def make_solver(N, Nrho, M, dev, Ne=8, K=3, dt=1e-3, scheme='imex-lm-bdf2',
                sphere='full', precision_mode=None):
    ini = couette_astd_ini(scheme=scheme, penalty='boltz-bgk-direct-gll',
                           Ne=Ne, K=K, Nv=N, Nrho=Nrho, M=M, dev=dev, dt=dt,
                           nsteps=10 ** 7, ic='maxwellian', noise=0.0,
                           sphere=sphere, precision_mode=precision_mode)
    return DGFSABstd1D(Config(ini))


def _profiles(m):
    # bulk moments (Nqr, Ne, 10): shear stress P:xy (8), heat flux Q:x (4)
    return m[..., 8].ravel(), m[..., 4].ravel()


def _rel_profile_diff(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def experiment(N=32, Nrho=16, M=12, dev=6.0, dt=1e-3, sphere='full',
               steady_tol=1e-8,
               max_steps=40000, n_maxwellian=20000, harvest_steps=3000,
               harvest_every=10, train_steps=40000, train_time=300.0, k=10,
               tol=1e-3, seed=20261203, check_every=10):
    out = dict(config=dict(N=N, Nrho=Nrho, M=M, L=dev, Ne=8, K=3, dt=dt,
                           scheme='imex-lm-bdf2', steady_tol=steady_tol, k=k,
                           tol=tol))
    plain = make_solver(N, Nrho, M, dev, dt=dt, sphere=sphere)
    rp = st.run_to_steady(plain, steady_tol, max_steps, check_every)
    pxy_p, qx_p = _profiles(rp['moments'])
    out['plain'] = dict(steps=rp['steps'], wall_s=rp['wall_s'],
                        residual=rp['residual'])
    op = plain.sm._op
    c0, L = plain.vm.c0(), plain.vm.L()
    # training data
    t0 = time.time()
    fm = st.perturbed_maxwellians(c0, n_maxwellian, seed)
    hs = make_solver(N, Nrho, M, dev, dt=dt, sphere=sphere)
    fh = st.harvest(hs, harvest_steps, harvest_every)
    fh = torch.cat([fh, plain.u.reshape(-1, plain.u.shape[-1])])
    f_all = torch.cat([fm, fh])
    del fm, fh
    q_all = st.operator_pairs(op, f_all)
    torch.cuda.synchronize()
    out['data'] = dict(pairs=int(f_all.shape[0]), maxwellian=n_maxwellian,
                       harvested=int(f_all.shape[0]) - n_maxwellian,
                       seconds=time.time() - t0)
    net = FNOSurrogate(N, L, q_scale=1.0, max_batch=24, seed=seed % 1000)
    t0 = time.time()
    hist = st.train(net, f_all, q_all, train_steps, batch=24, lr=2e-3,
                    time_budget=train_time, log_every=250,
                    tail=out['data']['harvested'], tail_frac=0.5)
    torch.cuda.synchronize()
    out['training'] = dict(steps=hist[-1][0], seconds=time.time() - t0,
                           loss_first=hist[0][1], loss_last=hist[-1][1])
    del f_all, q_all
    # held-out residuals
    fm_test = st.perturbed_maxwellians(c0, 48, seed + 1)
    out['residual_heldout_maxwellian_median'] = float(
        np.median(st.residuals(net, op, fm_test)))
    out['residual_steady_couette_median'] = float(
        np.median(st.residuals(net, op, plain.u.reshape(-1, plain.u.shape[-1]))))
    # the solver with the fused FP32 operator in place of the FP64 one (no
    # surrogate)
    f32 = make_solver(N, Nrho, M, dev, dt=dt, sphere=sphere, precision_mode='fp32')
    rf = st.run_to_steady(f32, steady_tol, max_steps, check_every)
    pxy, qx = _profiles(rf['moments'])
    out['fp32-fused-operator'] = dict(
        steps=rf['steps'], wall_s=rf['wall_s'], residual=rf['residual'],
        speedup_vs_plain=rp['wall_s'] / rf['wall_s'],
        shear_stress_rel_diff=_rel_profile_diff(pxy, pxy_p),
        heat_flux_rel_diff=_rel_profile_diff(qx, qx_p))
    del f32
    # surrogate-assisted runs: the plain operator (FP64, or the fused FP32
    # operator) checks every k-th call and serves as the fallback
    for mode, correct, prec in (('surrogate', False, None),
                                ('surrogate+defect', True, None),
                                ('surrogate+defect, fp32 checks', True, 'fp32')):
        sol = make_solver(N, Nrho, M, dev, dt=dt, sphere=sphere, precision_mode=prec)
        hook = st.SurrogateBoltzmann(sol, net, k=k, tol=tol, correct=correct)
        sol.boltzmann = hook
        rs = st.run_to_steady(sol, steady_tol, max_steps, check_every)
        pxy, qx = _profiles(rs['moments'])
        out[mode] = dict(steps=rs['steps'], wall_s=rs['wall_s'],
                         residual=rs['residual'],
                         speedup_vs_plain=rp['wall_s'] / rs['wall_s'],
                         speedup_vs_fp32_plain=rf['wall_s'] / rs['wall_s'],
                         shear_stress_rel_diff=_rel_profile_diff(pxy, pxy_p),
                         heat_flux_rel_diff=_rel_profile_diff(qx, qx_p),
                         **hook.stats())
        del sol, hook
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--quick', action='store_true')
    args = ap.parse_args()
    from . import build
    build.build()
    if args.quick:
        rep = experiment(N=16, Nrho=8, M=6, dev=5.0, dt=2e-3, sphere='auto',
                         steady_tol=1e-6, check_every=1,
                         max_steps=3000, n_maxwellian=512, harvest_steps=200,
                         harvest_every=10, train_steps=400, train_time=30.0)
    else:
        rep = experiment()
    print(json.dumps(rep))


if __name__ == '__main__':
    main()
