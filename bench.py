"""Benchmark of the fused fast-spectral collision operator Q(f,f) on B200.

Workload: the batched FP32 VHS configuration -- 24 spatial points (Ne=8,
K=3), velocity grid N=32^3 on [-6,6]^3, full-sphere M=12 design, Nrho=16,
omega=0.81 -- with seeded synthetic Couette-like distributions (Maxwellians
with u_y in [-0.1,0.1], T in [0.95,1.05], times 1 +- 1% uniform noise).
One step = one batched evaluation of Q(f,f) at all 24 points (one RHS stage).

Prints one JSON line (rank 0).  ``--impl reference`` times the CPU oracle
(the reference algorithm restated in NumPy/SciPy, all host cores) instead.
Multi-GPU (torchrun): every rank evaluates its own 24 points (weak scaling,
no data-path collective); time is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(workload='vhs-couette-fp32-batched', N=32, M=12, Nrho=16,
                L=6.0, points=24, Ne=8, K=3, omega=0.81, sphere='full-12pt',
                parallelism='points sharded over ranks (weak)',
                l2='flushed between timed steps (256 MB write)')
METRIC = 'Q(f,f) evals/s at N=32^3 (FP32 fused, M=12, Nrho=16, 24 points)'
UNIT = 'evals/s'


def make_inputs(rank=0):
    from dgfs1d_gpu_b200.workloads import couette_distributions, vhs_mesh_params
    prm = vhs_mesh_params(32, 12, 16, 6., True)
    f = couette_distributions(prm['c0'], 24, seed=20261203 + rank)
    return prm, f


def max_over_ranks(torch, dist, value, world, device):
    """The maximum of a per-rank float over all ranks (the job's time)."""
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, world, ms_max):
    """Whole-job throughput: every rank's units over the slowest rank's time
    (weak scaling: each rank evaluates its own points)."""
    return units_per_rank * world / (ms_max * 1e-3)


def cpu_oracle_rate(prm, f, budget_s=12.0, max_evals=4):
    """Evals/s of the oracle (CPU checker) on this host's cores, bounded."""
    from oracle.collision import VHSTables, vhs_gll_fs
    tab = VHSTables(prm['N'], prm['L'], prm['qz'], prm['qw'], prm['sz'],
                    prm['sw'], prm['gamma'],
                    sphere_factor=prm['sphere_factor'])
    prefac = prm['prefac']
    vhs_gll_fs(tab, prefac, f[0])  # warm-up
    t0 = time.perf_counter()
    n = 0
    while n < max_evals and (n == 0 or time.perf_counter() - t0 < budget_s):
        vhs_gll_fs(tab, prefac, f[n % len(f)])
        n += 1
    dt = time.perf_counter() - t0
    return n / dt, n, dt


class ClockSampler:
    """nvidia-smi clock/throttle sampling (every 100 ms) over the bench's
    timed regions."""
    Q = ('clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
         'clocks_event_reasons.hw_slowdown,'
         'clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,'
         'clocks_event_reasons.sw_power_cap')

    def __init__(self, device_index):
        self.idx = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.idx), '--query-gpu=' + self.Q,
                 '--format=csv,noheader,nounits', '-lms', '100'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self
        # wait for the first sample so the timed region is covered
        import select
        r, _, _ = select.select([self.proc.stdout], [], [], 5.0)
        self.first = self.proc.stdout.readline() if r else ''
        return self

    def __exit__(self, *a):
        self.rows = []
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        for line in (getattr(self, 'first', '') + out).strip().splitlines():
            parts = [p.strip() for p in line.split(',')]
            if len(parts) >= 8:
                self.rows.append(parts)

    def summary(self):
        if not getattr(self, 'rows', None):
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['unsampled']}
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        rows = [r for r in self.rows if num(r[0]) is not None]
        mx = [num(r[1]) for r in rows if num(r[1]) is not None]
        pw = [num(r[2]) or 0.0 for r in rows]
        # under load: power at least half of the run's maximum
        hot = [r for r, p in zip(rows, pw) if pw and p >= 0.5 * max(pw)]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown',
                 'sw_power_cap']
        reasons = sorted({names[i] for r in hot for i in range(4)
                          if r[4 + i].lower() == 'active'})
        return {'sm_mhz': float(np.median([num(r[0]) for r in hot]))
                if hot else None,
                'sm_max_mhz': max(mx) if mx else None,
                'reasons': reasons, 'samples': len(rows),
                'samples_under_load': len(hot),
                'power_w_max': max(pw) if pw else None}


def fp32_fma_peak(torch):
    """Measured FP32 FMA throughput (TFLOP/s) of this GPU, own kernel."""
    from dgfs1d_gpu_b200 import _native as nat
    import ctypes
    L = nat.lib()
    out = ctypes.c_double(0)
    nat.check(L.dgfs_fma_peak(ctypes.byref(out), ctypes.c_void_p(
        torch.cuda.current_stream().cuda_stream)))
    return out.value


def run_reference(args, rank, world):
    """CPU oracle arm: rank 0 only, all host cores.  One step is a bounded
    sample of the 24-point workload: 2 of its points, evaluated one after
    another (the reference's serial per-point loop, std.py:352-356); the line
    reports the measured time per step and the rate in evals/s."""
    if rank != 0:
        return
    prm, f = make_inputs(0)
    cores = os.cpu_count() or 1
    from oracle.collision import VHSTables, vhs_gll_fs
    tab = VHSTables(prm['N'], prm['L'], prm['qz'], prm['qw'], prm['sz'],
                    prm['sw'], prm['gamma'],
                    sphere_factor=prm['sphere_factor'])
    per_step = 2
    k = 0

    def step():
        nonlocal k
        for _ in range(per_step):
            vhs_gll_fs(tab, prm['prefac'], f[k % len(f)])
            k += 1
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    value = args.steps * per_step / dt
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': UNIT,
        'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': 1e3 * dt / args.steps, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
        'data': 'synthetic', 'config': dict(WORKLOAD),
        'cpu_baseline': {'value': value, 'unit': UNIT, 'cores': cores,
                         'kind': 'port',
                         'sample': f'each step = {per_step} of the 24 points, '
                                   'one NumPy/SciPy oracle evaluation each '
                                   '(reference algorithm, 3T+3 FFTs per eval, '
                                   'complex128, scipy.fft '
                                   f'workers={cores}); {args.steps} steps'},
        'e2e': {'value': value, 'unit': UNIT, 'h2d_bytes_per_step': 0,
                'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)


def surrogate_line(torch, prm, fd, op32, op64, timed, args):
    from dgfs1d_gpu_b200.surrogate import FNOSurrogate
    from dgfs1d_gpu_b200 import surrogate_train as st
    import time as _t
    net = FNOSurrogate(32, prm['L'], q_scale=1.0, max_batch=24, seed=5)
    t0 = _t.time()
    fm = st.perturbed_maxwellians(prm['c0'], 4096, 20261203)
    # Couette-like states: the bench family with other seeds
    from dgfs1d_gpu_b200.workloads import couette_distributions
    fc = torch.tensor(np.concatenate([couette_distributions(prm['c0'], 24, seed=s)
                                      for s in range(64)]), device='cuda')
    f_tr = torch.cat([fm, fc])
    q_tr = st.operator_pairs(op32, f_tr)
    hist = st.train(net, f_tr, q_tr, 100000, batch=24, lr=2e-3,
                    time_budget=args.surrogate_train_s, log_every=500,
                    tail=fc.shape[0], tail_frac=0.5)
    train_s = _t.time() - t0
    del fm, fc, f_tr, q_tr
    Qs = torch.zeros_like(fd)
    net.eval(fd, Qs)
    Q64 = torch.zeros_like(fd)
    op64.eval(fd, Q64)
    torch.cuda.synchronize()
    err = float(torch.linalg.norm(Qs - Q64) / torch.linalg.norm(Q64))
    Q = torch.zeros_like(fd)
    ms = timed(lambda: net.eval(fd, Q), max(3, args.steps // 4), 3)
    return {'value': fd.shape[0] / (ms * 1e-3), 'unit': UNIT, 'ms_per_step': ms,
            'err_vs_fp64_rel_l2': err, 'dtype': 'bf16 (FP32 accumulate)',
            'train_seconds': train_s, 'train_steps': hist[-1][0],
            'train_loss_last': hist[-1][1],
            'train_pairs': '4096 perturbed Maxwellians + 1536 Couette-like states',
            'tensor_cores': 'tcgen05.mma kind::f16 (dense layers, projection)',
            'error_flag': net.device_error(), '_net': net}


def couette_segment_line(torch, net, warm=300, nsteps=300, k=10, tol=1e-3):
    """The learned part inside a run: the IMEX Couette solver (Kn 0.1,
    diffuse walls u_y = -/+0.1, N=32, M=12, Nrho=16, Ne=8, K=3,
    imex-lm-bdf2, dt=1e-3, the fused FP32 operator) advanced `warm` steps
    from rest, then `nsteps` more steps three ways from that same state:
    the plain operator (the method without the surrogate), the surrogate
    plus the defect of its last check, and the surrogate alone between
    checks (the plain operator checks every k-th call and serves every call
    while a check is above tol).  Wall time of the segment and the shear
    stress / heat flux profiles against the plain segment."""
    import time as _t
    from dgfs1d_gpu_b200.surrogate_couette import (make_solver, _profiles,
                                                   _rel_profile_diff)
    from dgfs1d_gpu_b200 import surrogate_train as st
    out = {'workload': 'IMEX Couette Kn=0.1, N=32, M=12, Nrho=16, Ne=8, K=3, '
                       'imex-lm-bdf2, dt=1e-3, FP32 operator; segment after '
                       f'{warm} steps from rest', 'warm_steps': warm,
           'steps': nsteps, 'k': k, 'tol': tol}
    ref = None
    for mode in ('plain', 'surrogate+defect', 'surrogate'):
        sol = make_solver(32, 16, 12, 6.0, precision_mode='fp32')
        for _ in range(warm):
            sol.step()
        hook = None
        if mode != 'plain':
            hook = st.SurrogateBoltzmann(sol, net, k=k, tol=tol,
                                         correct=mode == 'surrogate+defect')
            sol.boltzmann = hook
        torch.cuda.synchronize()
        t0 = _t.perf_counter()
        for _ in range(nsteps):
            sol.step()
        torch.cuda.synchronize()
        wall = _t.perf_counter() - t0
        pxy, qx = _profiles(sol.bulk_moments())
        rec = {'wall_s': wall, 'ms_per_step': 1e3 * wall / nsteps}
        if ref is None:
            ref = (wall, pxy, qx)
        else:
            rec.update(gain_vs_plain=ref[0] / wall,
                       shear_stress_rel_diff=_rel_profile_diff(pxy, ref[1]),
                       heat_flux_rel_diff=_rel_profile_diff(qx, ref[2]),
                       **hook.stats())
        out[mode] = rec
        del sol, hook
    return out


def _rel_l2(torch, a, b):
    return float(torch.linalg.norm((a - b).double()) /
                 torch.linalg.norm(b.double()))


def _moment_errors(m32, m64):
    """Per-field error of (Nqr, Ne, 10) moments: max over points of
    |m32 - m64| / max |m64| for rho, U:y, T, Q:x, P:xy."""
    from dgfs1d_gpu_b200.std.moments import FIELDS
    out = {}
    for name in ('rho', 'U:y', 'T', 'Q:x', 'P:xy'):
        k = FIELDS.index(name)
        scale = np.max(np.abs(m64[..., k]))
        out[name] = float(np.max(np.abs(m32[..., k] - m64[..., k])) / scale) \
            if scale > 0 else 0.0
    return out


def _solver_pair(torch, ini32, ini64):
    from dgfs1d_gpu_b200.config import Config
    from dgfs1d_gpu_b200.std.solver import DGFSStd1D
    s32, s64 = DGFSStd1D(Config(ini32)), DGFSStd1D(Config(ini64))
    if not torch.equal(s32.u, s64.u):
        raise RuntimeError('FP32 and FP64 runs must start from the same state')
    return s32, s64


def _run_ms(torch, sol, nsteps):
    """CUDA-event time of nsteps solver steps (graph replays), no L2 flush:
    a solver run keeps its state resident."""
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(nsteps):
        sol.step()
    e.record()
    e.synchronize()
    return s.elapsed_time(e)


def stress_line(torch, timed, args):
    """The stress-size operator: hard spheres (omega = 0.5), N=48^3 on
    [-8,8]^3, full-sphere M=32 design, Nrho=24, 96 points (Ne=32, K=3), FP32
    mode, seeded Couette-like distributions; error against the FP64 operator
    on the same inputs (both with the conservation projection)."""
    from dgfs1d_gpu_b200.collision import VHSOperator
    from dgfs1d_gpu_b200.workloads import couette_distributions, vhs_mesh_params
    prm = vhs_mesh_params(48, 32, 24, 8.0, True, omega=0.5)
    f = torch.tensor(couette_distributions(prm['c0'], 96, seed=7), device='cuda')
    op = VHSOperator(**prm, precision='fp32', max_evals=96)
    op.set_projection(True)
    Q = torch.zeros_like(f)
    ms = timed(lambda: op.eval(f, Q), 5, 3)
    Q.zero_()
    op.eval(f, Q)
    op.close()
    op64 = VHSOperator(**prm, precision='fp64', max_evals=16)
    op64.set_projection(True)
    Q64 = torch.zeros_like(f)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    op64.eval(f, Q64)
    t1.record()
    t1.synchronize()
    err = _rel_l2(torch, Q, Q64)
    op64.close()
    out = {'workload': 'HS, N=48, L=8, M=32 full sphere, Nrho=24, 96 points, '
                       'FP32 + FP64 projection',
           'value': 96 / (ms * 1e-3), 'unit': UNIT, 'ms_per_step': ms,
           'fp64_ms_per_step': t0.elapsed_time(t1),
           'err_vs_fp64_rel_l2': err,
           'finite': bool(torch.isfinite(Q).all())}
    del f, Q, Q64
    return out


def fp64_n48_line(torch, timed, args):
    """The FP64 operator at N=48, the grid and rule of the reference's Lax
    examples (M=6 half sphere, Nrho=6, on [-10, 10]^3), 24
    points, seeded Couette-like distributions."""
    from dgfs1d_gpu_b200.collision import VHSOperator
    from dgfs1d_gpu_b200.workloads import couette_distributions, vhs_mesh_params
    prm = vhs_mesh_params(48, 6, 6, 10.0, False)
    f = torch.tensor(couette_distributions(prm['c0'], 24, seed=9), device='cuda')
    op = VHSOperator(**prm, precision='fp64', max_evals=24)
    Q = torch.zeros_like(f)
    ms = timed(lambda: op.eval(f, Q), 5, 3)
    op.close()
    del f, Q
    return {'workload': 'VHS, N=48, M=6 half sphere, Nrho=6, 24 points, FP64',
            'value': 24 / (ms * 1e-3), 'unit': UNIT, 'ms_per_step': ms,
            'err_vs_fp64_rel_l2': 0.0}


def stress_solver_line(torch, timed, args, nseg=2):
    """Steps of the stress configuration's solver: Mach-1.5 normal shock of
    hard spheres, N=48^3 on [-8,8]^3, M=32, Nrho=24, Ne=32, K=3 (96 points),
    inlet boundaries, lse-rk45 (5 RHS stages per step), FP32 operator, one
    CUDA graph per step; then an nseg-step segment of the same solver with
    the FP32 and the FP64 operator from the same state, compared."""
    from dgfs1d_gpu_b200.configs import normal_shock_std_ini
    s32, s64 = _solver_pair(torch, normal_shock_std_ini(precision_mode='fp32'),
                            normal_shock_std_ini(precision_mode='fp64'))
    s32.capture_step()
    ms = timed(s32.step, 3, 1)
    s32.u.copy_(s64.u)
    ms32 = _run_ms(torch, s32, nseg)
    ms64 = _run_ms(torch, s64, nseg)
    err = _rel_l2(torch, s32.u, s64.u)
    merr = _moment_errors(s32.bulk_moments(), s64.bulk_moments())
    ok = bool(torch.isfinite(s32.u).all())
    out = {'workload': 'normal shock Mach 1.5, HS, N=48, M=32, Nrho=24, '
                       'Ne=32, K=3, lse-rk45, FP32 operator, graph per step',
           'ms_per_step': ms, 'evals_per_s': 5 * 96 / (ms * 1e-3),
           'projected_s_for_500_steps': 500 * ms * 1e-3,
           'segment_steps': nseg, 'segment_ms_fp32': ms32,
           'segment_ms_fp64_eager': ms64,
           'err_vs_fp64_rel_l2': err, 'moment_err_vs_fp64': merr,
           'finite': ok}
    del s32, s64
    return out


def solver_line(torch, timed, args, nsteps=200):
    """The batched FP32 Couette configuration as a run: dgfsStd1D, N=32,
    M=12, Nrho=16, Ne=8, K=3, 200 ssp-rk3 steps (three RHS stages of 24
    point evaluations each), one CUDA graph per step; the same 200 steps
    with the plain FP64 operator from the same initial state, and the FP32
    run's error against it."""
    from dgfs1d_gpu_b200.configs import couette_c2_ini
    s32, s64 = _solver_pair(torch, couette_c2_ini('fp32', nsteps),
                            couette_c2_ini('fp64', nsteps))
    n = max(3, args.steps // 10)
    ms_eager = timed(s32.step, n, 3)
    s32.u.copy_(s64.u)
    s32.t, s32.nacptsteps = s64.t, 0
    s32.capture_step()
    s64.capture_step()
    ms32 = _run_ms(torch, s32, nsteps)
    ms64 = _run_ms(torch, s64, nsteps)
    m32, m64 = s32.bulk_moments(), s64.bulk_moments()
    evals = 3 * 24
    out = {'workload': 'dgfsStd1D Couette, N=32, M=12, Nrho=16, Ne=8, K=3, '
                       'ssp-rk3, FP32 operator, u_y -0.1..0.1 and T 0.95..1.05 '
                       'across x, 1% noise, dt=1.25e-4',
           'steps': nsteps, 'ms_per_step_graph': ms32 / nsteps,
           'ms_per_step_eager': ms_eager,
           'fp64_ms_per_step_graph': ms64 / nsteps,
           'run_s_fp32': ms32 * 1e-3, 'run_s_fp64': ms64 * 1e-3,
           'speedup_fp32_vs_fp64': ms64 / ms32,
           'evals_per_s_graph': evals * nsteps / (ms32 * 1e-3),
           'graph_launches_per_step': 1,
           'err_vs_fp64_rel_l2': _rel_l2(torch, s32.u, s64.u),
           'moment_err_vs_fp64': _moment_errors(m32, m64)}
    del s32, s64
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=200)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='native', choices=['native', 'reference'])
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-surrogate', action='store_true')
    ap.add_argument('--surrogate-train-s', type=float, default=40.0)
    ap.add_argument('--kernel-only', action='store_true',
                    help='run only warm-up + timed FP32 evaluations (for ncu '
                         'launch lists); prints ms per step')
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get('RANK', 0))
    world = int(os.environ.get('WORLD_SIZE', 1))
    local = int(os.environ.get('LOCAL_RANK', 0))

    if args.impl == 'reference':
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    from dgfs1d_gpu_b200 import build
    if rank == 0 or not os.path.exists(build.OUT):
        build.build()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device('cuda', local))
    from dgfs1d_gpu_b200.collision import VHSOperator

    prm, f = make_inputs(rank)
    E = f.shape[0]
    fd = torch.tensor(f, dtype=torch.float64, device='cuda')
    op32 = VHSOperator(**prm, precision='fp32', max_evals=E)
    op64 = VHSOperator(**prm, precision='fp64', max_evals=E)
    Q = torch.zeros_like(fd)
    flush = torch.empty(64 * 2 ** 20, dtype=torch.float32, device='cuda')

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        barrier()
        tot = 0.0
        for _ in range(steps):
            flush.fill_(1.0)  # evict L2 (256 MB > 126 MB) outside the events
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record()
            fn()
            e.record()
            e.synchronize()
            tot += s.elapsed_time(e)
        barrier()
        return max_over_ranks(torch, dist, tot, world, 'cuda') / steps

    if args.kernel_only:
        ms = timed(lambda: op32.eval(fd, Q), args.steps, args.warmup)
        if rank == 0:
            print(json.dumps({'kernel_only_ms_per_step': ms}), flush=True)
        return

    # clocks sampled over the whole native run (every timed region below)
    clk = ClockSampler(local).__enter__()

    # project autotuner: cluster size of the FP32 terms kernel, timed on this
    # very batch
    tune = op32.autotune(fd, Q, reps=3)

    # headline: FP32 fused operator, inputs resident in HBM, one evaluation
    # as one CUDA graph launch (its kernels and stream forks captured once);
    # the plain FP64 path (same kernels, FP64 arithmetic, no split) the same
    # way; the eager launch sequences beside them
    from dgfs1d_gpu_b200.batch import StageGraph
    g32 = StageGraph([lambda: op32.eval(fd, Q)])
    g32.capture()
    g64 = StageGraph([lambda: op64.eval(fd, Q)])
    g64.capture()
    ms32 = timed(g32.replay, args.steps, args.warmup)
    ms64 = timed(g64.replay, max(3, args.steps // 2), 3)
    ms32_eager = timed(lambda: op32.eval(fd, Q), args.steps, args.warmup)
    ms64_eager = timed(lambda: op64.eval(fd, Q), max(3, args.steps // 2), 3)
    del g32, g64

    # error of the FP32 mode vs the FP64 mode on this workload
    Q32 = torch.zeros_like(fd)
    Q64 = torch.zeros_like(fd)
    op32.eval(fd, Q32)
    op64.eval(fd, Q64)
    torch.cuda.synchronize()
    err = _rel_l2(torch, Q32, Q64)

    # end to end through the C ABI with host buffers: every step copies its
    # 24 distributions from pinned host memory to the device and its Q back.
    # (1) one step at a time: H2D f, eval, D2H Q on one stream;
    fh = torch.tensor(f, dtype=torch.float64).pin_memory()
    qh = [torch.empty_like(fh).pin_memory() for _ in range(2)]
    fdev = [torch.empty_like(fd) for _ in range(2)]
    qdev = [torch.empty_like(fd) for _ in range(2)]

    def e2e_step():
        fdev[0].copy_(fh, non_blocking=True)
        qdev[0].zero_()
        op32.eval(fdev[0], qdev[0])
        qh[0].copy_(qdev[0], non_blocking=True)

    ms_e2e_seq = timed(e2e_step, args.steps, args.warmup)

    # (2) a stream of steps, as a solver feeding batches of points through
    # the operator runs it: double-buffered device arrays on three streams,
    # so that step i+1's H2D and step i-1's D2H overlap step i's evaluation;
    # the 256 MB L2 flush precedes every evaluation on the compute stream
    s_in, s_cmp, s_out = (torch.cuda.Stream() for _ in range(3))
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_cmp = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]

    def e2e_stream(nsteps):
        for i in range(nsteps):
            b = i % 2
            with torch.cuda.stream(s_in):
                if i >= 2:
                    s_in.wait_event(ev_cmp[b])    # step i-2 has read fdev[b]
                fdev[b].copy_(fh, non_blocking=True)
                ev_in[b].record(s_in)
            with torch.cuda.stream(s_cmp):
                s_cmp.wait_event(ev_in[b])
                if i >= 2:
                    s_cmp.wait_event(ev_out[b])   # qdev[b] of step i-2 is out
                flush.fill_(1.0)
                qdev[b].zero_()
                op32.eval(fdev[b], qdev[b])
                ev_cmp[b].record(s_cmp)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_cmp[b])
                qh[b].copy_(qdev[b], non_blocking=True)
                ev_out[b].record(s_out)

    e2e_stream(args.warmup)
    barrier()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(s_in)
    e2e_stream(args.steps)
    t_end.record(s_out)
    t_end.synchronize()
    barrier()
    ms_e2e = max_over_ranks(torch, dist, t_start.elapsed_time(t_end), world,
                            'cuda') / args.steps
    # the streamed results equal the resident-input evaluation
    Qchk = torch.zeros_like(fd)
    op32.eval(fd, Qchk)
    torch.cuda.synchronize()
    e2e_match = bool(torch.equal(qh[(args.steps - 1) % 2].cuda(), Qchk))

    # per-kernel durations inside the timed region: CUDA events recorded by
    # the library on the launching stream between its kernels
    from dgfs1d_gpu_b200 import _native as nat
    import ctypes
    nat.check(nat.lib().dgfs_vhs_profile(op32._h, 1))
    stage = np.zeros(5)
    buf = (ctypes.c_double * 5)()
    for _ in range(args.warmup):
        op32.eval(fd, Q)
    for _ in range(args.steps):
        flush.fill_(1.0)
        op32.eval(fd, Q)
        nat.check(nat.lib().dgfs_vhs_stage_ms(op32._h, buf))
        stage += np.array(buf[:])
    stage /= args.steps
    nat.check(nat.lib().dgfs_vhs_profile(op32._h, 0))
    terms_ms = float(stage[3])

    fma_peak = fp32_fma_peak(torch)

    solver = solver_line(torch, timed, args)
    stress = stress_line(torch, timed, args)
    fp64_n48 = fp64_n48_line(torch, timed, args)
    stress_solver = stress_solver_line(torch, timed, args)
    # learned surrogate (FNO, BF16 tensor-core dense layers): trained here for
    # a bounded time on operator pairs, then timed and compared with FP64
    sur = None
    if not args.no_surrogate:
        sur = surrogate_line(torch, prm, fd, op32, op64, timed, args)
        sur['couette_segment'] = couette_segment_line(torch, sur.pop('_net'))

    # uneven multi-problem batch: 6 VHS problems (N=16/24/32) + 2 VSS
    # mixtures.  Merged: the problems that share an operator evaluated in
    # one call per kernel (one group per N, one for the mixtures), the
    # groups as concurrent branches of one CUDA graph per stage; against the
    # per-problem calls issued one after another on one stream and against
    # the per-problem graph; error against the same problems in FP64
    from dgfs1d_gpu_b200.batch import StageGraph
    from dgfs1d_gpu_b200.workloads_c3 import build_c3
    groups = build_c3(precision='fp32', merged=True, autotune=True)
    members = [m for g in groups for m in g['members']]
    b_evals = sum(g['nevals'] for g in groups)
    b_steps = max(3, args.steps // 4)
    sg = StageGraph([g['fn'] for g in groups])
    sg.capture()
    ms_graph = timed(sg.replay, b_steps, 3)
    del sg
    sg = None
    probs = build_c3(precision='fp32')

    def serial():
        for p in probs:
            p['fn']()
    ms_serial = timed(serial, b_steps, 3)
    sg1 = StageGraph([p['fn'] for p in probs])
    sg1.capture()
    ms_graph1 = timed(sg1.replay, b_steps, 3)
    del sg1
    for g in groups:
        g['fn']()
    probs64 = build_c3(precision='fp64')
    for p in probs64:
        p['fn']()
    torch.cuda.synchronize()
    b_err = {}
    # the merged groups list their members by group (grouped by N), not in
    # the problems' own order: pair each with its FP64 twin by name
    by_name = {p['name']: p for p in probs64}
    for a in members:
        b = by_name[a['name']]
        qa = a['Q'] if isinstance(a['Q'], list) else [a['Q']]
        qb = b['Q'] if isinstance(b['Q'], list) else [b['Q']]
        b_err[a['name']] = max(_rel_l2(torch, x, y) for x, y in zip(qa, qb))
    batch = {'value': b_evals * world / (ms_graph * 1e-3), 'unit': UNIT,
             'ms_per_stage': ms_graph, 'graph_launches_per_stage': 1,
             'groups': [g['name'] for g in groups],
             'autotuned_variants': {g['name']: g.get('variant') for g in groups
                                    if 'variant' in g},
             'serial_stream_ms_per_stage': ms_serial,
             'per_problem_graph_ms_per_stage': ms_graph1,
             'speedup_vs_serial_stream': ms_serial / ms_graph,
             'problems': [m['name'] for m in members],
             'evals_per_stage': b_evals,
             'err_vs_fp64_rel_l2': b_err,
             'note': 'VSS evals count each (p,q) pair at each point; '
                     'serial = one call per problem, one after another'}
    del groups, probs, probs64

    barrier()
    clk.__exit__(None, None, None)
    if rank == 0:
        peaks = {}
        pth = os.path.join(ROOT, 'MEASURED_PEAKS.json')
        if os.path.exists(pth):
            peaks = json.load(open(pth))
        hbm_peak = peaks.get('hbm_gbs', 6650.0)
        peak_src = 'measured' if 'hbm_gbs' in peaks else 'fallback'
        n = 32 ** 3
        Nrho, Mu, M = 16, 6, 12
        T = M * Nrho
        fft = 5 * n * np.log2(n)
        # minimal exact algorithm per evaluation (the unit of work):
        # 2T + Nrho + 3 transforms of n points and ~20 flops per point and
        # term of pointwise work: 1.116 GFLOP at this configuration
        min_flops_eval = (2 * T + Nrho + 3) * fft + 20 * T * n
        # flops per terms-kernel launch as executed: Mu*Nrho packed inverse
        # and Nrho/2 packed forward 3-D FFTs, ~40 flops per point and term
        exec_flops = E * ((Mu * Nrho + Nrho // 2) * fft + Mu * Nrho * n * 40)
        # compulsory HBM bytes per evaluation of the fused operator: read f,
        # read and write Q (FP64 arrays)
        compulsory = 3 * n * 8
        evals = E * world
        # DRAM bytes per launch of the terms kernel from the committed ncu
        # summary (dram__bytes_read.sum + dram__bytes_write.sum, one capture)
        traffic = None
        tp = os.path.join(ROOT, 'profiles', 'vhs_terms_fp32_n32_24pts.md')
        if os.path.exists(tp):
            import re
            txt = open(tp).read()
            rd = re.search(r'dram__bytes_read\.sum \| ([0-9.]+) MB', txt)
            wr = re.search(r'dram__bytes_write\.sum \| ([0-9.]+) MB', txt)
            if rd and wr:
                traffic = (float(rd.group(1)) + float(wr.group(1))) * 1e6
        cores = os.cpu_count() or 1
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            rate, ns, dt = cpu_oracle_rate(prm, f, budget_s=12.0,
                                           max_evals=48)
            cpu = {'value': rate, 'unit': UNIT, 'cores': cores, 'kind': 'port',
                   'sample': f'{ns} single-point evals ({dt:.1f} s) of the '
                             'NumPy/SciPy oracle of this workload '
                             f'(complex128, scipy.fft workers={cores})'}
        value = job_rate(E, world, ms32)
        achieved = value / world * min_flops_eval / 1e12
        clocks = clk.summary()
        line = {
            'metric': METRIC,
            'value': value,
            'unit': UNIT,
            'n_gpus': world,
            'steps': args.steps,
            'warmup': args.warmup,
            'ms_per_step': ms32,
            'higher_is_better': True,
            'scaling': 'weak',
            'vs_baseline': None,
            'dtype': 'f32',
            'data': 'synthetic',
            'config': dict(WORKLOAD),
            'fp64_plain': {'value': evals / (ms64 * 1e-3), 'unit': UNIT,
                           'ms_per_step': ms64,
                           'ms_per_step_eager': ms64_eager},
            'speedup_fp32_vs_fp64': ms64 / ms32,
            'ms_per_step_eager': ms32_eager,
            'speedup_fp32_vs_fp64_eager': ms64_eager / ms32_eager,
            'step': 'one 24-point evaluation as one CUDA graph launch',
            'err_fp32_vs_fp64_rel_l2': err,
            'e2e': {'value': evals / (ms_e2e * 1e-3), 'unit': UNIT,
                    'h2d_bytes_per_step': int(fh.numel() * 8),
                    'd2h_bytes_per_step': int(qh[0].numel() * 8),
                    'ms_per_step': ms_e2e,
                    'mode': 'stream of steps through dgfs_vhs_eval: pinned '
                            'host f -> device, evaluation, Q -> pinned host '
                            'every step, double-buffered on three streams '
                            '(H2D of step i+1 and D2H of step i-1 overlap '
                            'step i), L2 flushed before every evaluation',
                    'result_equals_resident_eval': e2e_match,
                    'one_step_at_a_time': {
                        'value': evals / (ms_e2e_seq * 1e-3), 'unit': UNIT,
                        'ms_per_step': ms_e2e_seq}},
            'roofline': {
                'bound': 'fp32-fma',
                'kernel': f'vhs_terms_fp32_kernel<32,{op32.variant}> '
                          '(dominant) within the whole operator',
                'achieved': achieved, 'peak': fma_peak, 'unit': 'TFLOP/s',
                'frac': achieved / fma_peak,
                'flops_per_eval_minimal_algorithm': min_flops_eval,
                'frac_executed': exec_flops / (terms_ms * 1e-3) / 1e12 / fma_peak,
                'executed_flops_per_terms_launch': exec_flops,
                'launch_ms': terms_ms,
                'peak_source': 'measured in this run by dgfs_fma_peak (own '
                               'FP32 FMA kernel, every SM); MEASURED_PEAKS.json '
                               'has no FP32 figure',
                'peak_clock_sm_mhz': clocks.get('sm_mhz'),
                'traffic': traffic,
                'hbm': {'traffic_per_terms_launch': traffic,
                        'achieved_gbs': (traffic / (terms_ms * 1e-3) / 1e9
                                         if traffic else None),
                        'peak_gbs': hbm_peak, 'peak_source': peak_src,
                        'frac': (traffic / (terms_ms * 1e-3) / 1e9 / hbm_peak
                                 if traffic else None),
                        'compulsory_bytes_per_step': compulsory * E,
                        'traffic_over_compulsory': (traffic / (compulsory * E)
                                                    if traffic else None)}},
            'stage_ms': dict(zip(['prologue', 'tables', 'maxwell_gain',
                                  'terms', 'epilogue'],
                                 [round(float(x), 4) for x in stage])),
            'uneven_batch': batch,
            'surrogate': sur,
            'solver_step': solver,
            'stress_n48': stress,
            'fp64_n48': fp64_n48,
            'stress_solver_n48': stress_solver,
            'autotune_terms_ms': {str(k): round(v, 4) for k, v in tune.items()},
            'terms_cluster': op32.variant,
            'cpu_baseline': cpu,
            'clocks': clocks,
            'gpu_launches': 6 * args.steps,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
