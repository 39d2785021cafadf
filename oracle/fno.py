"""CPU FP64 forward/backward of the FNO surrogate (test infrastructure only).

Test infrastructure only (see ``oracle/__init__.py``): the checker of the
CUDA surrogate kernels (``dgfs1d_gpu_b200/csrc/fno_kernels.cuh``).  The
surrogate is a new component with no counterpart in the reference, so this
module is its defining restatement: the network, the loss and the exact
gradients in float64 NumPy.  Features: [f/rho, g, g r, g r^2] with
g = (f - M)/(rho sigma), sigma = rms((f - M)/rho), r = |c - u|/sqrt(T);
output scale rho^2 sigma q_scale.  With ``emulate_bf16`` the activations that the
GPU stores in BF16 (features, v_l, y_l, the spectral output U) are rounded the same way, so that the
two agree to FP32-accumulation differences; without it the module is a plain
float64 network, which ``tests/test_fno_oracle.py`` pins against central
finite differences.

Parameter layout (flat float32, same order as ``fno::Layout``):
P[4][32], p[32]; for l in 0..3: W_l[K^3][32][32] complex (re, im), D_l[32][32],
d_l[32]; Q1[32][128], q1[128], q2[128], q2b[1].
"""
import numpy as np

WD, PJ, CIN = 32, 128, 4


def layout(K):
    o, L = 0, {}

    def take(name, size):
        nonlocal o
        L[name] = (o, size)
        o += size
    take('P', CIN * WD)
    take('p', WD)
    for l in range(4):
        take(f'W{l}', 2 * K ** 3 * WD * WD)
        take(f'D{l}', WD * WD)
        take(f'd{l}', WD)
    take('Q1', WD * PJ)
    take('q1', PJ)
    take('q2', PJ)
    take('q2b', 1)
    L['total'] = o
    return L


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64).reshape(a.shape)


def modes(K):
    return np.array([k if k < K // 2 else k - K for k in range(K)])


def tables(N, K):
    """F[k][x] = exp(-2 pi i k x / N) for the retained modes."""
    x = np.arange(N)
    return np.exp(-2j * np.pi * np.outer(modes(K), x) / N)


# GELU in the tanh form (Hendrycks & Gimpel): x/2 (1 + tanh(c (x + a x^3)))
_GC, _GA = np.sqrt(2.0 / np.pi), 0.044715


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(_GC * (x + _GA * x ** 3)))


def gelu_d(x):
    t = np.tanh(_GC * (x + _GA * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * _GC * (1.0 + 3.0 * _GA * x * x)


class FNO:
    """The surrogate network on an N^3 grid with K modes per axis."""

    def __init__(self, N, K, L, q_scale, params, emulate_bf16=True):
        self.N, self.K, self.Lbox, self.sQ = N, K, L, q_scale
        self.lay = layout(K)
        w = np.asarray(params)
        w = bf16(w) if emulate_bf16 else w.astype(np.float64)
        self.w = {k: w[v[0]:v[0] + v[1]] for k, v in self.lay.items()
                  if k != 'total'}
        self.emu = emulate_bf16
        self.F = tables(N, K)
        self.c0 = np.linspace(-L + L / N, L - L / N, N)
        self.cw = (2.0 * L / N) ** 3

    def _r(self, x):
        return bf16(x) if self.emu else x

    def W(self, l):
        K = self.K
        a = self.w[f'W{l}'].reshape(K ** 3, WD, WD, 2)
        return a[..., 0] + 1j * a[..., 1]

    # separable truncated transforms on [B, N, N, N, C] <-> [B, K, K, K, C]
    def dft(self, v, F):
        t = np.einsum('kx,bxyzc->bkyzc', F, v)
        t = np.einsum('ky,bxyzc->bxkzc', F, t)
        return np.einsum('kz,bxyzc->bxykc', F, t)

    def idft(self, u, G):
        t = np.einsum('xk,bkyzc->bxyzc', G, u)
        t = np.einsum('yk,bxkzc->bxyzc', G, t)
        return np.einsum('zk,bxykc->bxyzc', G, t)

    def features(self, f):
        N, c0, cw = self.N, self.c0, self.cw
        B = f.shape[0]
        g = np.meshgrid(c0, c0, c0, indexing='ij')
        cv = np.stack([x.ravel() for x in g])
        rho = f.sum(1) * cw
        u = (f @ cv.T) * cw / rho[:, None]
        e = (f @ (cv ** 2).sum(0)) * cw / rho
        T = (2.0 / 3.0) * (e - (u ** 2).sum(1))
        r2 = ((cv[None] - u[:, :, None]) ** 2).sum(1) / T[:, None]
        M = (rho / (np.pi * T) ** 1.5)[:, None] * np.exp(-r2)
        gq = (f - M) / rho[:, None]
        sig = np.maximum(np.sqrt((gq * gq).mean(1)), 1e-300)
        gq = gq / sig[:, None]
        x0 = np.stack([f / rho[:, None], gq, gq * np.sqrt(r2), gq * r2], axis=-1)
        return self._r(x0).reshape(B, N, N, N, CIN), rho ** 2 * sig

    def forward(self, f):
        """f: [B, N^3] float64.  Returns the network output [B, N^3] and a
        cache for backward."""
        w, N, K = self.w, self.N, self.K
        x0, qs = self.features(f)
        B = f.shape[0]
        v = [self._r(x0 @ w['P'].reshape(CIN, WD) + w['p'])]
        y, Vh = [], []
        G = np.conj(self.F).T / N
        for l in range(4):
            V = self.dft(v[l], self.F)
            Vh.append(V)
            Uh = np.einsum('bmi,mio->bmo', V.reshape(B, K ** 3, WD), self.W(l))
            U = self._r(self.idft(Uh.reshape(B, K, K, K, WD), G).real)
            yl = self._r(v[l] @ w[f'D{l}'].reshape(WD, WD) + w[f'd{l}'] + U)
            y.append(yl)
            v.append(self._r(gelu(yl)) if l < 3 else yl)
        z = v[4] @ w['Q1'].reshape(WD, PJ) + w['q1']
        out = gelu(z) @ w['q2'] + w['q2b'][0]
        cache = dict(x0=x0, v=v, y=y, Vh=Vh, z=z, qs=qs)
        return out.reshape(B, -1), cache

    def loss(self, out, Qt, qs):
        t = Qt / (qs * self.sQ)[:, None]
        e = out - t
        tn = (t * t).sum(1)
        L = (e * e).sum(1) / tn
        dout = 2.0 * e / (out.shape[0] * tn[:, None])
        return L, dout

    def backward(self, dout, cache):
        """Gradients of sum(dout * out) w.r.t. every parameter (flat)."""
        w, N, K = self.w, self.N, self.K
        v, y, Vh, z = cache['v'], cache['y'], cache['Vh'], cache['z']
        B = dout.shape[0]
        g = {}
        do = dout.reshape(B, N, N, N, 1)
        a = gelu(z)
        dz = do * w['q2'] * gelu_d(z)
        g['q2'] = (do * a).reshape(-1, PJ).sum(0)
        g['q2b'] = np.array([do.sum()])
        g['Q1'] = (v[4].reshape(-1, WD).T @ dz.reshape(-1, PJ)).ravel()
        g['q1'] = dz.reshape(-1, PJ).sum(0)
        dv = dz @ w['Q1'].reshape(WD, PJ).T
        Fs = self.F / N               # B^H per axis (adjoint of the IDFT)
        Gs = np.conj(self.F).T        # A^H per axis (adjoint of the DFT)
        for l in range(3, -1, -1):
            dy = dv * gelu_d(y[l]) if l < 3 else dv
            g[f'D{l}'] = (v[l].reshape(-1, WD).T @ dy.reshape(-1, WD)).ravel()
            g[f'd{l}'] = dy.reshape(-1, WD).sum(0)
            dvl = dy @ w[f'D{l}'].reshape(WD, WD).T
            gU = self.dft(dy, Fs).reshape(B, K ** 3, WD)
            V = Vh[l].reshape(B, K ** 3, WD)
            gW = np.einsum('bmi,bmo->mio', np.conj(V), gU)
            g[f'W{l}'] = np.stack([gW.real, gW.imag], axis=-1).ravel()
            gV = np.einsum('bmo,mio->bmi', gU, np.conj(self.W(l)))
            dvl = dvl + self.idft(gV.reshape(B, K, K, K, WD), Gs).real
            dv = dvl
        x0 = cache['x0']
        g['P'] = (x0.reshape(-1, CIN).T @ dv.reshape(-1, WD)).ravel()
        g['p'] = dv.reshape(-1, WD).sum(0)
        flat = np.zeros(self.lay['total'])
        for k, sl in self.lay.items():
            if k != 'total':
                flat[sl[0]:sl[0] + sl[1]] = g[k]
        return flat
