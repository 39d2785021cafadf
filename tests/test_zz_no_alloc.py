"""The allocation-free Q(f,f) entry point, checked against the handle path.

Some callers of this library cannot allocate device memory: services whose
device memory is a fixed pool handed out at start-up, plugins loaded into
processes that forbid cudaMalloc once serving has begun, and time loops that
cannot afford cudaMalloc's implicit device synchronisation.
dgfs_vhs_eval_noalloc serves them
from a static device array inside the library.  This file is named so that
pytest collects it last; it runs correctly alone or after the other tests.
"""
import ctypes

import numpy as np
import pytest
import torch

from dgfs1d_gpu_b200 import _native as nat
from dgfs1d_gpu_b200.workloads import couette_distributions, vhs_mesh_params

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-11   # relative L2, the FP64 tolerance of the parity tests


def _desc(prm, keep):
    arrs = [np.ascontiguousarray(prm['qz'], dtype=np.float64),
            np.ascontiguousarray(prm['qw'], dtype=np.float64),
            np.ascontiguousarray(np.asarray(prm['sz']).ravel(), dtype=np.float64),
            np.ascontiguousarray(prm['c0'], dtype=np.float64)]
    keep.extend(arrs)
    ptr = [ctypes.cast(a.ctypes.data, ctypes.POINTER(ctypes.c_double))
           for a in arrs]
    d = nat.VhsDesc()
    d.N, d.Nrho, d.M = prm['N'], len(arrs[0]), len(arrs[2]) // 3
    d.L = prm['L']
    d.qz, d.qw, d.sz, d.c0 = ptr
    d.sw, d.sphere_factor = prm['sw'], prm['sphere_factor']
    d.gamma, d.prefac, d.sinc_eps = prm['gamma'], prm['prefac'], 1e-15
    d.cw = prm['cw']
    d.precision = nat.DGFS_PREC_FP64
    d.max_evals = 1
    return d


def _noalloc(d, f, Q, nevals):
    return nat.lib().dgfs_vhs_eval_noalloc(
        ctypes.byref(d), ctypes.c_void_p(f.data_ptr()),
        ctypes.c_void_p(Q.data_ptr()), None, 0, None, 0, nevals,
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


@pytest.mark.parametrize('case', [(8, 6, 4, 5., False, 3),
                                  (16, 6, 8, 5., False, 5),
                                  (32, 12, 16, 6., True, 2)],
                         ids=['N8', 'N16', 'N32'])
def test_noalloc_matches_handle_path_twice(case):
    from dgfs1d_gpu_b200 import build
    build.build()
    from dgfs1d_gpu_b200.collision import VHSOperator
    N, M, Nrho, dev, full, nev = case
    prm = vhs_mesh_params(N, M, Nrho, dev, full)
    f = torch.tensor(couette_distributions(prm['c0'], nev), device='cuda')
    op = VHSOperator(**prm, precision='fp64', max_evals=nev)
    Qref = torch.zeros_like(f)
    op.eval(f, Qref)
    keep = []
    d = _desc(prm, keep)
    for _ in range(2):   # two calls in a row share the static scratch
        Q = torch.zeros_like(f)
        nat.check(_noalloc(d, f, Q, nev))
        torch.cuda.synchronize()
        err = float(torch.linalg.norm(Q - Qref) / torch.linalg.norm(Qref))
        assert err < FP64_TOL, err


def test_noalloc_rejects_shapes_beyond_its_scratch():
    prm = vhs_mesh_params(32, 12, 32, 6., True)   # Nrho=32 at N=32: too big
    keep = []
    d = _desc(prm, keep)
    f = torch.zeros(32 ** 3, dtype=torch.float64, device='cuda')
    Q = torch.zeros_like(f)
    rc = _noalloc(d, f, Q, 1)
    assert rc == -4   # DGFS_ERR_CAPACITY
    assert b'allocation-free maximum' in nat.lib().dgfs_last_error_string()
