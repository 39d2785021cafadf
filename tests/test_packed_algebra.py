"""The exact algebra behind the FP32 terms kernel, checked in float64 NumPy.

The kernel (vhs_terms_fp32_kernel / vhs_nyq_planes_kernel) replaces the
reference's two inverse transforms per (p, q) term -- IFFT(cos a F) and
IFFT(sin a F), std/scattering.py:251-313, vhs-gll.mako:101-218 -- by one
packed complex transform of (cos a + sin a)-type multipliers plus three 2-D
transforms of the Nyquist planes, splits f = M + g, and packs two radial
points into one forward transform.  This test restates that sequence with
full 3-D NumPy transforms and compares it with the oracle's literal
restatement of the reference: the identity must hold to rounding.
"""
import numpy as np
import pytest

from oracle.collision import vhs_gll_fs
from tests._cases import vhs_case, vhs_tables


def _packed_q(tab, prefac, f, cv):
    N, n = tab.N, tab.n
    l0 = np.array([i if i < N // 2 else i - N for i in range(N)], float)
    LX, LY, LZ = np.meshgrid(l0, l0, l0, indexing='ij')
    inv = lambda X: np.fft.ifftn(X) * n
    fwd = np.fft.fftn
    f3 = f.reshape(N, N, N)
    F = fwd(f3) / n
    w = (2 * tab.L / N) ** 3
    rho = f.sum() * w
    u = (cv * f).sum(1) * w / rho
    T = (((cv - u[:, None]) ** 2).sum(0) * f).sum() * w / (1.5 * rho)
    M = (rho / (np.pi * T) ** 1.5
         * np.exp(-((cv - u[:, None]) ** 2).sum(0) / T)).reshape(N, N, N)
    FM = fwd(M) / n
    Fg = F - FM
    Nrho, Mfull = tab.aa.shape[:2]
    sz = tab.sz
    used, uq, mult = [False] * Mfull, [], []
    for q in range(Mfull):          # antipodal pairs merged, weight 2
        if used[q]:
            continue
        used[q], m = True, 1
        for r in range(q + 1, Mfull):
            if not used[r] and np.all(sz[r] == -sz[q]):
                used[r], m = True, 2
                break
        uq.append(q)
        mult.append(m)
    b1w = (tab.sphere_factor * tab.qw * tab.sw / n)[:, None] * tab.bb1
    nyq = [(L == -N // 2) for L in (LX, LY, LZ)]
    GM = np.zeros((N, N, N), complex)   # Maxwellian gain (FP64 on the GPU)
    for p in range(Nrho):
        acc = np.zeros((N, N, N), complex)
        for q in range(Mfull):
            a = tab.aa[p, q].reshape(N, N, N)
            t3, t4 = inv(np.cos(a) * FM), inv(np.sin(a) * FM)
            acc += t3 * t3 + t4 * t4
        GM += b1w[p].reshape(N, N, N) * fwd(acc)
    S = []
    for p in range(Nrho):
        Sp = np.zeros((N, N, N))
        for qi, q in enumerate(uq):
            kap = np.pi / tab.L * tab.qz[p] / 2 * sz[q]
            ph = kap[0] * LX + kap[1] * LY + kap[2] * LZ
            sc = np.sqrt(mult[qi])
            E = sc * np.exp(1j * ph)
            fS = np.ones((N, N, N), complex)
            for ax in range(3):
                fS = np.where(nyq[ax], fS * np.exp(1j * kap[ax] * N), fS)
            m = (E * (1 + fS) * (1 - 1j) / 2).real
            mc = (E * (1 - fS) * (1 - 1j) / 2).real
            assert np.all(mc[~(nyq[0] | nyq[1] | nyq[2])] == 0)
            z, zc = inv(m * Fg), inv(mc * Fg)
            C, s, sR, cI = z.real, z.imag, zc.real, zc.imag
            um = inv(E * FM)
            vm = inv(sc * np.exp(-1j * ph) * FM)
            A, B = um + vm, um - vm
            Sp += (C * (A.real + C) + s * (B.real - s) + sR * (B.imag + sR)
                   - cI * (A.imag + cI))
        S.append(Sp)
    H = np.zeros((N, N, N), complex)
    for p in range(0, Nrho, 2):
        S1 = S[p + 1] if p + 1 < Nrho else 0 * S[p]
        b1 = b1w[p + 1].reshape(N, N, N) if p + 1 < Nrho else 0
        H += (b1w[p].reshape(N, N, N) - 1j * b1) * fwd(S[p] + 1j * S1)
    G = inv(GM + H).real
    fL = inv(tab.bb2.reshape(N, N, N) * F).real
    return (prefac * (G - f3 * fL)).ravel()


@pytest.mark.parametrize('case', [(8, 6, 4, 5., False), (16, 6, 8, 5., False),
                                  (16, 12, 7, 5., True)],
                         ids=['N8', 'N16', 'N16-full-odd-Nrho'])
def test_packed_transforms_equal_reference_sequence(case):
    N, M, Nrho, dev, full = case
    vm, prefac, gamma, f = vhs_case(N, M, Nrho, dev, full, nslots=1,
                                    noise=0.05)
    tab = vhs_tables(vm, gamma)
    ref = vhs_gll_fs(tab, prefac, f[0])
    new = _packed_q(tab, prefac, f[0], vm.cv)
    assert np.linalg.norm(new - ref) / np.linalg.norm(ref) < 1e-12
