"""The CPU FP64 FNO oracle (the checker of the surrogate's CUDA kernels),
pinned against central finite differences of its own loss, and its parameter
layout against the library's."""
import numpy as np
import pytest

from oracle import fno as ofno


def _maxwellians(N, L, B, seed):
    rng = np.random.default_rng(seed)
    c0 = np.linspace(-L + L / N, L - L / N, N)
    g = np.meshgrid(c0, c0, c0, indexing='ij')
    cv = np.stack([x.ravel() for x in g])
    f = np.empty((B, N ** 3))
    for b in range(B):
        rho, T = rng.uniform(0.5, 2.0), rng.uniform(0.7, 1.5)
        u = rng.uniform(-0.3, 0.3, 3)
        m = rho / (np.pi * T) ** 1.5 * np.exp(-((cv - u[:, None]) ** 2).sum(0) / T)
        f[b] = m * (1 + 0.05 * rng.uniform(-1, 1, m.shape))
    return f


def test_layout_matches_library():
    from dgfs1d_gpu_b200.surrogate import layout
    for K in (4, 8, 12):
        assert layout(K) == ofno.layout(K)


def test_oracle_gradient_matches_finite_differences():
    from dgfs1d_gpu_b200.surrogate import init_params
    N, K, L, B = 8, 4, 5.0, 2
    w = init_params(K, seed=3).astype(np.float64)
    f = _maxwellians(N, L, B, seed=4)
    Qt = np.random.default_rng(5).standard_normal((B, N ** 3)) * 1e-2

    def loss(wv):
        net = ofno.FNO(N, K, L, 0.5, wv, emulate_bf16=False)
        out, cache = net.forward(f)
        Lb, dout = net.loss(out, Qt, cache['qs'])
        return Lb.mean(), net, dout, cache

    _, net, dout, cache = loss(w)
    g = net.backward(dout, cache)
    lay = ofno.layout(K)
    rng = np.random.default_rng(6)
    for name in ('P', 'p', 'W0', 'D0', 'd0', 'W2', 'D3', 'Q1', 'q1', 'q2', 'q2b'):
        o, s = lay[name]
        for j in rng.choice(s, size=min(3, s), replace=False):
            h = 1e-5 * max(1.0, abs(w[o + j]))
            wp, wm = w.copy(), w.copy()
            wp[o + j] += h
            wm[o + j] -= h
            fd = (loss(wp)[0] - loss(wm)[0]) / (2 * h)
            assert abs(fd - g[o + j]) <= 1e-6 * max(abs(fd), 1e-3), (name, j, fd, g[o + j])
