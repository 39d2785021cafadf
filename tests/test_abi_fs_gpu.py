"""The per-point entry dgfs_vhs_fs, bound with plain ctypes the way a
maintainer would bind it inside the reference's DGFSVHSGLLScatteringModelStd
(the descriptor mirror and the call of the binding shown for
std/scattering.py:51-313), checked against the oracle.

The reference's driver calls fs(d_f, d_g, d_Q, elem, modein, modeout) once
per (element, mode) (dgfs1D/std/std.py:352-356); the kernel reads slot
modein*Ne + elem and accumulates into slot modeout*Ne + elem
(vhs-gll.mako:399-433).  The test uses elem > 0 and modein != modeout, so a
wrong slot mapping or a missing += shows."""
import ctypes

import numpy as np
import pytest
import torch

from oracle.collision import VHSTables, vhs_gll_fs
from tests._cases import vhs_case

pytestmark = pytest.mark.gpu


class _VhsDesc(ctypes.Structure):            # mirrors dgfs_vhs_desc
    _dp = ctypes.POINTER(ctypes.c_double)
    _fields_ = [('N', ctypes.c_int32), ('Nrho', ctypes.c_int32), ('M', ctypes.c_int32),
                ('L', ctypes.c_double), ('qz', _dp), ('qw', _dp), ('sz', _dp),
                ('sw', ctypes.c_double), ('sphere_factor', ctypes.c_double),
                ('gamma', ctypes.c_double), ('prefac', ctypes.c_double),
                ('sinc_eps', ctypes.c_double), ('cw', ctypes.c_double), ('c0', _dp),
                ('precision', ctypes.c_int32), ('max_evals', ctypes.c_int32)]


@pytest.fixture(scope='module')
def lib():
    from dgfs1d_gpu_b200 import build
    path = build.build()
    return ctypes.CDLL(path)      # a plain binding, not the package's


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_fs_slot_arithmetic_matches_oracle(lib, precision):
    K, Ne = 3, 4
    vm, prefac, gamma, f = vhs_case(16, 6, 8, 5., False, nslots=K * Ne)
    fp64 = precision == 'fp64'
    # the reference's sinc regulariser: 1e-15 in double, 1e-6 in float
    # (vhs-gll.mako:9-23); the oracle tables use the same one
    eps = 1e-15 if fp64 else 1e-6
    tab = VHSTables(vm.Nv, vm.L, vm.qz, vm.qw, vm.sz, vm.sw, gamma,
                    sphere_factor=vm.sphere_factor, eps=eps)
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
    arrs = [np.ascontiguousarray(x, np.float64) for x in
            (vm.qz, vm.qw, np.asarray(vm.sz).ravel(), vm.cv[2, :vm.Nv])]
    d = _VhsDesc(vm.Nv, len(vm.qz), len(arrs[2]) // 3, vm.L, *map(dp, arrs[:3]),
                 vm.sw, vm.sphere_factor, gamma, prefac, eps, vm.cw, dp(arrs[3]),
                 0 if fp64 else 1, K * Ne)
    h = ctypes.c_void_p()
    assert lib.dgfs_vhs_create(ctypes.byref(d), ctypes.byref(h)) == 0, \
        lib.dgfs_last_error_string()
    try:
        dt = torch.float64 if fp64 else torch.float32
        fd = torch.tensor(f, dtype=dt, device='cuda')
        Q0 = (torch.randn(f.shape, dtype=torch.float64) * 1e-4).to(dt).cuda()
        Q = Q0.clone()
        calls = [(1, 0, 2), (3, 2, 1), (2, 1, 1)]    # (elem, modein, modeout)
        for elem, mi, mo in calls:
            rc = lib.dgfs_vhs_fs(h, ctypes.c_void_p(fd.data_ptr()),
                                 ctypes.c_void_p(Q.data_ptr()), 1 if fp64 else 0,
                                 Ne, elem, mi, mo, None)
            assert rc == 0, lib.dgfs_last_error_string()
        torch.cuda.synchronize()
        got = (Q.double() - Q0.double()).cpu().numpy()
        exp = np.zeros_like(f)
        fin = fd.double().cpu().numpy()
        for elem, mi, mo in calls:
            exp[mo * Ne + elem] += vhs_gll_fs(tab, prefac, fin[mi * Ne + elem])
        # the FP32 mode is checked at its 1e-5 bound; the FP32 arrays add
        # their own rounding of Q0 + dQ, far below it
        tol = 1e-11 if fp64 else 1e-5
        touched = sorted({mo * Ne + elem for elem, _, mo in calls})
        for s in range(K * Ne):
            if s in touched:
                err = np.linalg.norm(got[s] - exp[s]) / np.linalg.norm(exp[s])
                assert err < tol, (s, err)
            else:
                assert np.array_equal(Q[s].cpu().numpy(), Q0[s].cpu().numpy()), s
        # bad element / mode arguments are refused before any launch
        assert lib.dgfs_vhs_fs(h, ctypes.c_void_p(fd.data_ptr()),
                               ctypes.c_void_p(Q.data_ptr()), 1 if fp64 else 0,
                               Ne, Ne, 0, 0, None) == -1
    finally:
        lib.dgfs_vhs_destroy(h)
