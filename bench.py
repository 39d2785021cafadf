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
                L=6.0, points=24, Ne=8, K=3, omega=0.81, sphere='full-12pt')
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
    """nvidia-smi clock/throttle sampling during the timed region."""
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
        sm = [float(r[0]) for r in self.rows if r[0].replace('.', '').isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown',
                 'sw_power_cap']
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if r[4 + i].lower() == 'active'})
        return {'sm_mhz': float(np.median(sm)) if sm else None,
                'sm_max_mhz': max(mx) if mx else None,
                'reasons': reasons, 'samples': len(self.rows)}


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
    """CPU oracle arm: rank 0 only, all host cores."""
    if rank != 0:
        return
    prm, f = make_inputs(0)
    cores = os.cpu_count() or 1
    rates = []
    for _ in range(args.warmup):
        cpu_oracle_rate(prm, f, budget_s=2.0, max_evals=1)
    t_all = 0.0
    n_all = 0
    for _ in range(args.steps):
        r, n, dt = cpu_oracle_rate(prm, f, budget_s=6.0, max_evals=2)
        rates.append(r)
        t_all += dt
        n_all += n
    value = n_all / t_all
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': UNIT,
        'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': 1e3 * 24 / value, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
        'data': 'synthetic', 'config': dict(WORKLOAD),
        'cpu_baseline': {'value': value, 'unit': UNIT, 'cores': cores,
                         'kind': 'port',
                         'sample': f'{n_all} single-point evals of the NumPy/'
                                   'SciPy oracle (reference algorithm, 3T+3 '
                                   'FFTs per eval, complex128, '
                                   f'scipy.fft workers={cores})'},
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
            'error_flag': net.device_error()}


def stress_line(torch, timed, args):
    """The stress-size operator: hard spheres (omega = 0.5), N=48^3 on
    [-8,8]^3, full-sphere M=32 design, Nrho=24, 96 points (Ne=32, K=3), FP32
    mode, seeded Couette-like distributions."""
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
    torch.cuda.synchronize()
    ok = bool(torch.isfinite(Q).all())
    op.close()
    del f, Q
    return {'workload': 'HS, N=48, L=8, M=32 full sphere, Nrho=24, 96 points, '
                        'FP32 + FP64 projection',
            'value': 96 / (ms * 1e-3), 'unit': UNIT, 'ms_per_step': ms,
            'finite': ok}


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
            'value': 24 / (ms * 1e-3), 'unit': UNIT, 'ms_per_step': ms}


def stress_solver_line(torch, timed, args):
    """Steps of the stress configuration's solver: Mach-1.5 normal shock of
    hard spheres, N=48^3 on [-8,8]^3, M=32, Nrho=24, Ne=32, K=3 (96 points),
    inlet boundaries, lse-rk45 (5 RHS stages per step), FP32 operator, one
    CUDA graph per step."""
    from dgfs1d_gpu_b200.config import Config
    from dgfs1d_gpu_b200.configs import normal_shock_std_ini
    from dgfs1d_gpu_b200.std.solver import DGFSStd1D
    sol = DGFSStd1D(Config(normal_shock_std_ini()))
    sol.capture_step()
    ms = timed(sol.step, 3, 1)
    ok = bool(torch.isfinite(sol.u).all())
    return {'workload': 'normal shock Mach 1.5, HS, N=48, M=32, Nrho=24, '
                        'Ne=32, K=3, lse-rk45, FP32 operator, graph per step',
            'ms_per_step': ms, 'evals_per_s': 5 * 96 / (ms * 1e-3),
            'projected_s_for_500_steps': 500 * ms * 1e-3, 'finite': ok}


def solver_line(torch, timed, args):
    """The whole dgfsStd1D step on the batched FP32 Couette configuration
    (ssp-rk3: three RHS stages of 24 points each), eager and as one CUDA
    graph per step."""
    from dgfs1d_gpu_b200.config import Config
    from dgfs1d_gpu_b200.configs import couette_std_ini
    from dgfs1d_gpu_b200.std.solver import DGFSStd1D
    ini = couette_std_ini(Ne=8, K=3, Nv=32, Nrho=16, M=12, dev=6.0,
                          scheme='ssp-rk3', dt=2e-4, nsteps=200,
                          precision_mode='fp32', sphere='full')
    sol = DGFSStd1D(Config(ini))
    n = max(3, args.steps // 10)
    ms_eager = timed(sol.step, n, 3)
    sol.capture_step()
    ms_graph = timed(sol.step, n, 3)
    evals = 3 * 24
    return {'workload': 'dgfsStd1D Couette, N=32, M=12, Nrho=16, Ne=8, K=3, '
                        'ssp-rk3, FP32 operator',
            'ms_per_step_graph': ms_graph, 'ms_per_step_eager': ms_eager,
            'evals_per_s_graph': evals / (ms_graph * 1e-3),
            'graph_launches_per_step': 1}


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

    # project autotuner: cluster size of the FP32 terms kernel, timed on this
    # very batch
    tune = op32.autotune(fd, Q, reps=3)

    # headline: FP32 fused operator, inputs resident in HBM
    with ClockSampler(local) as clk:
        ms32 = timed(lambda: op32.eval(fd, Q), args.steps, args.warmup)
    # plain FP64 path (same kernels, FP64 arithmetic, no split)
    ms64 = timed(lambda: op64.eval(fd, Q), max(3, args.steps // 2), 3)

    # error of the FP32 mode vs the FP64 mode on this workload
    Q32 = torch.zeros_like(fd)
    Q64 = torch.zeros_like(fd)
    op32.eval(fd, Q32)
    op64.eval(fd, Q64)
    torch.cuda.synchronize()
    err = float(torch.linalg.norm(Q32 - Q64) / torch.linalg.norm(Q64))

    # end to end through the C ABI with host buffers: H2D f, eval, D2H Q
    fh = torch.tensor(f, dtype=torch.float64).pin_memory()
    qh = torch.empty_like(fh).pin_memory()
    fdev = torch.empty_like(fd)
    qdev = torch.empty_like(fd)

    def e2e_step():
        fdev.copy_(fh, non_blocking=True)
        qdev.zero_()
        op32.eval(fdev, qdev)
        qh.copy_(qdev, non_blocking=True)

    ms_e2e = timed(e2e_step, args.steps, args.warmup)

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

    # learned surrogate (FNO, BF16 tensor-core dense layers): trained here for
    # a bounded time on operator pairs, then timed and compared with FP64
    solver = solver_line(torch, timed, args)
    stress = stress_line(torch, timed, args)
    fp64_n48 = fp64_n48_line(torch, timed, args)
    stress_solver = stress_solver_line(torch, timed, args)
    sur = None
    if not args.no_surrogate:
        sur = surrogate_line(torch, prm, fd, op32, op64, timed, args)

    # uneven multi-problem batch: 6 VHS problems (N=16/24/32) + 2 VSS
    # mixtures, one CUDA graph launch per stage vs the same launches issued
    # one after another on one stream
    from dgfs1d_gpu_b200.batch import StageGraph
    from dgfs1d_gpu_b200.workloads_c3 import build_c3
    probs = build_c3(precision='fp32')
    sg = StageGraph([p['fn'] for p in probs])
    sg.capture()
    b_evals = sum(p['nevals'] for p in probs)
    b_steps = max(3, args.steps // 4)
    ms_graph = timed(sg.replay, b_steps, 3)

    def serial():
        for p in probs:
            p['fn']()
    ms_serial = timed(serial, b_steps, 3)
    batch = {'value': b_evals * world / (ms_graph * 1e-3), 'unit': UNIT,
             'ms_per_stage': ms_graph, 'graph_launches_per_stage': 1,
             'serial_stream_ms_per_stage': ms_serial,
             'problems': [p['name'] for p in probs],
             'evals_per_stage': b_evals,
             'note': 'VSS evals count each (p,q) pair at each point'}
    del sg

    barrier()
    if rank == 0:
        peaks = {}
        pth = os.path.join(ROOT, 'MEASURED_PEAKS.json')
        if os.path.exists(pth):
            peaks = json.load(open(pth))
        hbm_peak = peaks.get('hbm_gbs', 6650.0)
        peak_src = 'measured' if 'hbm_gbs' in peaks else 'fallback'
        n = 32 ** 3
        Nrho, Mu = 16, 6
        # terms kernel, per launch: per eval read F_g (n complex FP32) and the
        # Nyquist-plane transforms (Nrho*Mu*3*N^2 complex FP32), write the
        # packed radial-pair spectra H (Nrho/2 * n complex FP32); b1w
        # (Nrho*n FP32) once
        alg_bytes = E * (n * 8 + Nrho * Mu * 3 * 32 * 32 * 8 + Nrho // 2 * n * 8) \
            + Nrho * n * 4
        # flops per eval as executed: Mu*Nrho packed inverse and Nrho/2
        # packed forward 3-D FFTs (5 n log2 n each) + the pointwise combine
        # (~40 flops per point and term)
        fft = 5 * n * np.log2(n)
        alg_flops = E * ((Mu * Nrho + Nrho // 2) * fft + Mu * Nrho * n * 40)
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
        line = {
            'metric': METRIC,
            'value': job_rate(E, world, ms32),
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
            'config': dict(WORKLOAD, parallelism=f'points-sharded x{world}',
                           l2='flushed between timed steps (256 MB write)'),
            'fp64_plain': {'value': evals / (ms64 * 1e-3), 'unit': UNIT,
                           'ms_per_step': ms64},
            'speedup_fp32_vs_fp64': ms64 / ms32,
            'err_fp32_vs_fp64_rel_l2': err,
            'e2e': {'value': evals / (ms_e2e * 1e-3), 'unit': UNIT,
                    'h2d_bytes_per_step': int(fh.numel() * 8),
                    'd2h_bytes_per_step': int(qh.numel() * 8)},
            'roofline': {'bound': 'hbm', 'kernel': f'vhs_terms_fp32_kernel<32,{op32.variant}>',
                         'achieved': alg_bytes / (terms_ms * 1e-3) / 1e9,
                         'peak': hbm_peak, 'unit': 'GB/s',
                         'frac': alg_bytes / (terms_ms * 1e-3) / 1e9 / hbm_peak,
                         'traffic': traffic, 'peak_source': peak_src,
                         'launch_ms': terms_ms},
            'roofline_fp32': {'bound': 'fp32-fma',
                              'achieved': alg_flops / (terms_ms * 1e-3) / 1e12,
                              'peak': fma_peak, 'unit': 'TFLOP/s',
                              'frac': alg_flops / (terms_ms * 1e-3) / 1e12 / fma_peak,
                              'peak_source': 'measured by dgfs_fma_peak'},
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
            'clocks': clk.summary(),
            'gpu_launches': 6 * args.steps,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
