"""The CUDA FNO surrogate against the CPU FP64 oracle (oracle/fno.py):
forward output, loss and every parameter gradient; conservation and +=
semantics of the surrogate's Q; and that training on operator pairs lowers
the loss."""
import numpy as np
import pytest
import torch

from oracle import fno as ofno
from tests.test_fno_oracle import _maxwellians

pytestmark = pytest.mark.gpu

N, L, B = 16, 5.0, 2
K = 8
SQ = 0.05


@pytest.fixture(scope='module')
def built():
    from dgfs1d_gpu_b200 import build
    build.build()


def _data(seed=11):
    f = _maxwellians(N, L, B, seed)
    Qt = np.random.default_rng(seed + 1).standard_normal((B, N ** 3)) * 1e-3
    return f, Qt


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_loss_and_gradients_match_oracle(built):
    from dgfs1d_gpu_b200.surrogate import FNOSurrogate, layout
    net = FNOSurrogate(N, L, q_scale=SQ, max_batch=4, seed=7)
    f, Qt = _data()
    fd = torch.tensor(f, device='cuda')
    qd = torch.tensor(Qt, device='cuda')
    net.train_step(fd, qd, update=False)
    torch.cuda.synchronize()
    loss = net.last_loss(B)
    g = net.grads()
    ref = ofno.FNO(N, K, L, SQ, net.params(), emulate_bf16=True)
    out, cache = ref.forward(f)
    Lb, dout = ref.loss(out, Qt, cache['qs'])
    gr = ref.backward(dout, cache)
    assert np.allclose(loss, Lb, rtol=2e-3), (loss, Lb)
    errs = {}
    for name, sl in layout(K).items():
        if name == 'total':
            continue
        o, s = sl
        errs[name] = e = _rel(g[o:o + s], gr[o:o + s])
        assert e < 2e-2, f'{name}: gradient rel L2 {e:.3e} ({errs})'
    print('gradient rel L2 vs oracle:', {k: f'{v:.1e}' for k, v in errs.items()})


def test_eval_is_conservative_accumulating_and_matches_oracle(built):
    from dgfs1d_gpu_b200.surrogate import FNOSurrogate
    net = FNOSurrogate(N, L, q_scale=SQ, max_batch=4, seed=8)
    f, _ = _data(21)
    fd = torch.tensor(f, device='cuda')
    Q0 = torch.zeros_like(fd)
    net.eval(fd, Q0)
    Q1 = torch.full_like(fd, 0.25)
    net.eval(fd, Q1)
    torch.cuda.synchronize()
    q = Q0.cpu().numpy()
    assert np.allclose(Q1.cpu().numpy() - 0.25, q, rtol=0, atol=1e-15)
    ref = ofno.FNO(N, K, L, SQ, net.params(), emulate_bf16=True)
    out, cache = ref.forward(f)
    c0 = ref.c0
    g = np.meshgrid(c0, c0, c0, indexing='ij')
    cv = np.stack([x.ravel() for x in g])
    phi = np.vstack([np.ones(N ** 3), cv, (cv ** 2).sum(0)]) * ref.cw
    G = phi @ np.vstack([np.ones(N ** 3), cv, (cv ** 2).sum(0)]).T
    for b in range(B):
        raw = cache['qs'][b] * SQ * out[b]
        lam = np.linalg.solve(G, phi @ raw)
        proj = raw - lam @ np.vstack([np.ones(N ** 3), cv, (cv ** 2).sum(0)])
        assert _rel(q[b], proj) < 1e-2
        # conserved to rounding of the FP64 projection of the raw output
        scale = np.abs(phi) @ np.abs(raw)
        assert np.all(np.abs(phi @ q[b]) <= 1e-12 * scale)


def test_training_on_operator_pairs_lowers_the_loss(built):
    from dgfs1d_gpu_b200.collision import VHSOperator
    from dgfs1d_gpu_b200.surrogate import FNOSurrogate
    from dgfs1d_gpu_b200.workloads import vhs_mesh_params
    prm = vhs_mesh_params(N, 6, 8, L, False)
    op = VHSOperator(**prm, precision='fp64', max_evals=8)
    f = torch.tensor(_maxwellians(N, L, 8, 31), device='cuda')
    Qt = torch.zeros_like(f)
    op.eval(f, Qt)
    net = FNOSurrogate(N, L, q_scale=1.0, max_batch=8, seed=9)
    net.train_step(f, Qt, update=False)
    first = net.last_loss(8).mean()
    for _ in range(100):
        net.train_step(f, Qt, lr=3e-3)
    net.train_step(f, Qt, update=False)
    last = net.last_loss(8).mean()
    print(f'training loss {first:.3e} -> {last:.3e}')
    assert np.isfinite(last) and last < 0.5 * first, (first, last)


def test_tensor_core_layers_match_cuda_core_layers(built):
    """The tcgen05 dense/projection kernels against the CUDA-core kernels on
    the same network and inputs (eval path, N=16 and N=32)."""
    from dgfs1d_gpu_b200.surrogate import FNOSurrogate
    for n_, l_ in ((16, 5.0), (32, 6.0)):
        net = FNOSurrogate(n_, l_, q_scale=SQ, max_batch=4, seed=12)
        f = torch.tensor(_maxwellians(n_, l_, 3, 41), device='cuda')
        out = []
        for tc in (True, False):
            net.set_tensor_cores(tc)
            Q = torch.zeros_like(f)
            net.eval(f, Q)
            torch.cuda.synchronize()
            out.append(Q.cpu().numpy())
        assert net.device_error() == 0
        e = _rel(out[0], out[1])
        print(f'N={n_}: tensor cores vs CUDA cores rel L2 {e:.2e}')
        assert e < 2e-2, e


def test_fused_eval_matches_per_axis_passes(built):
    """The fused evaluation kernels (register-FFT spectral passes, yz inverse
    fused with the tensor-core dense layer) against the per-axis DFT passes
    that training uses, on the same network and inputs (N=16 and N=32)."""
    from dgfs1d_gpu_b200.surrogate import FNOSurrogate, layout
    for n_, l_ in ((16, 5.0), (32, 6.0)):
        net = FNOSurrogate(n_, l_, q_scale=SQ, max_batch=4, seed=13)
        # spectral weights scaled up so that the spectral path dominates the
        # layers (at initialisation it is a small correction)
        w = net.params()
        for l in range(4):
            o, sz = layout(net.K)[f'W{l}']
            w[o:o + sz] *= 30.0
        net.set_params(w)
        f = torch.tensor(_maxwellians(n_, l_, 3, 43), device='cuda')
        out = []
        for fused in (True, False):
            net.set_fused(fused)
            Q = torch.zeros_like(f)
            net.eval(f, Q)
            torch.cuda.synchronize()
            out.append(Q.cpu().numpy())
        assert net.device_error() == 0
        e = _rel(out[0], out[1])
        print(f'N={n_}: fused vs per-axis passes rel L2 {e:.2e}')
        assert e < 1e-2, e
