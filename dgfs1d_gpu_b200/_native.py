"""ctypes binding of the in-tree C-ABI library ``libdgfs_sm100.so``.

The library is built in place by ``dgfs1d_gpu_b200.build.build()`` (nvcc,
sm_100a).  There is no fallback: if the library is missing or a call fails,
the error is raised.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, 'libdgfs_sm100.so')

DGFS_OK = 0
DGFS_F32, DGFS_F64 = 0, 1
DGFS_PREC_FP64, DGFS_PREC_FP32 = 0, 1

_c_dp = ctypes.POINTER(ctypes.c_double)


class VhsDesc(ctypes.Structure):
    """Mirror of ``dgfs_vhs_desc`` (include/dgfs_sm100.h)."""
    _fields_ = [
        ('N', ctypes.c_int32), ('Nrho', ctypes.c_int32), ('M', ctypes.c_int32),
        ('L', ctypes.c_double),
        ('qz', _c_dp), ('qw', _c_dp), ('sz', _c_dp),
        ('sw', ctypes.c_double), ('sphere_factor', ctypes.c_double),
        ('gamma', ctypes.c_double), ('prefac', ctypes.c_double),
        ('sinc_eps', ctypes.c_double), ('cw', ctypes.c_double),
        ('c0', _c_dp),
        ('precision', ctypes.c_int32), ('max_evals', ctypes.c_int32),
    ]


class VssDesc(ctypes.Structure):
    """Mirror of ``dgfs_vss_desc`` (include/dgfs_sm100.h)."""
    _fields_ = [
        ('N', ctypes.c_int32), ('Nrho', ctypes.c_int32), ('M', ctypes.c_int32),
        ('Mpre', ctypes.c_int32), ('nspcs', ctypes.c_int32),
        ('L', ctypes.c_double), ('qz', _c_dp), ('qw', _c_dp), ('sz', _c_dp),
        ('sw', ctypes.c_double), ('szpre', _c_dp), ('masses', _c_dp),
        ('gamma', _c_dp), ('eta', _c_dp), ('prefac', _c_dp),
        ('max_evals', ctypes.c_int32), ('precision', ctypes.c_int32),
    ]


class DgDesc(ctypes.Structure):
    """Mirror of ``dgfs_dg_desc`` (include/dgfs_sm100.h)."""
    _fields_ = [
        ('K', ctypes.c_int32), ('Ne', ctypes.c_int32), ('N', ctypes.c_int32),
        ('Nqr', ctypes.c_int32),
        ('trL', _c_dp), ('trR', _c_dp), ('D', _c_dp), ('gLD', _c_dp),
        ('gRD', _c_dp), ('invjac', _c_dp), ('c0', _c_dp), ('im', _c_dp),
        ('cw', ctypes.c_double),
        ('bc_kind', ctypes.c_int32 * 2),
        ('bc_f0', _c_dp * 2),
        ('bc_ux', ctypes.c_double * 2),
    ]


class DgfsError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code, msg):
        super().__init__(f'dgfs_sm100 error {code}: {msg}')
        self.code = code


_lib = None

# (name, restype, argtypes) of every exported entry point
class FnoDesc(ctypes.Structure):
    """Mirrors dgfs_fno_desc."""
    _fields_ = [('N', ctypes.c_int32), ('modes', ctypes.c_int32),
                ('max_batch', ctypes.c_int32), ('L', ctypes.c_double),
                ('q_scale', ctypes.c_double)]


_SIGNATURES = [
    ('dgfs_version', ctypes.c_char_p, []),
    ('dgfs_last_error_string', ctypes.c_char_p, []),
    ('dgfs_vhs_create', ctypes.c_int,
     [ctypes.POINTER(VhsDesc), ctypes.POINTER(ctypes.c_void_p)]),
    ('dgfs_vhs_eval', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
      ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
      ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]),
    ('dgfs_vhs_fs', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
      ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
      ctypes.c_void_p]),
    ('dgfs_vhs_eval_multi', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
      ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
      ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]),
    ('dgfs_vhs_eval2', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
      ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
      ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]),
    ('dgfs_vhs_fs2', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
      ctypes.c_int32, ctypes.c_void_p]),
    ('dgfs_vhs_last_moments', ctypes.c_void_p, [ctypes.c_void_p]),
    ('dgfs_vhs_device_error', ctypes.c_int,
     [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    ('dgfs_vhs_set_projection', ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    ('dgfs_vhs_variants', ctypes.c_int,
     [ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32]),
    ('dgfs_vhs_set_variant', ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    ('dgfs_fno_create', ctypes.c_int,
     [ctypes.POINTER(FnoDesc), ctypes.POINTER(ctypes.c_void_p)]),
    ('dgfs_fno_destroy', ctypes.c_int, [ctypes.c_void_p]),
    ('dgfs_fno_num_params', ctypes.c_int64, [ctypes.c_void_p]),
    ('dgfs_fno_set_params', ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ('dgfs_fno_get_params', ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ('dgfs_fno_get_grads', ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ('dgfs_fno_eval', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
      ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
      ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]),
    ('dgfs_fno_train_step', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
      ctypes.c_float, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]),
    ('dgfs_fno_last_loss', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32]),
    ('dgfs_fno_set_tensor_cores', ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    ('dgfs_fno_set_fused', ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    ('dgfs_fno_error', ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    ('dgfs_vhs_destroy', ctypes.c_int, [ctypes.c_void_p]),
    ('dgfs_vhs_profile', ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    ('dgfs_vhs_stage_ms', ctypes.c_int,
     [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    ('dgfs_fma_peak', ctypes.c_int,
     [ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    ('dgfs_vss_create', ctypes.c_int,
     [ctypes.POINTER(VssDesc), ctypes.POINTER(ctypes.c_void_p)]),
    ('dgfs_vss_destroy', ctypes.c_int, [ctypes.c_void_p]),
    ('dgfs_vss_eval', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
      ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
      ctypes.c_int32, ctypes.c_void_p]),
    ('dgfs_vss_eval_species_multi', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
      ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
      ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]),
    ('dgfs_vss_eval_species', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p),
      ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
      ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
      ctypes.c_void_p]),
    ('dgfs_dg_create', ctypes.c_int,
     [ctypes.POINTER(DgDesc), ctypes.POINTER(ctypes.c_void_p)]),
    ('dgfs_dg_destroy', ctypes.c_int, [ctypes.c_void_p]),
    ('dgfs_dg_advect', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
      ctypes.c_void_p]),
    ('dgfs_dg_wall_density', ctypes.c_int,
     [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    ('dgfs_dg_limit_positivity', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    ('dgfs_std_esbgk_relax', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
      ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
      ctypes.c_void_p]),
    ('dgfs_dg_set_entropy_stable', ctypes.c_int,
     [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    ('dgfs_dg_set_upwind', ctypes.c_int,
     [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
      ctypes.POINTER(ctypes.c_double), ctypes.c_int32]),
    ('dgfs_dg_set_wall_state', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
      ctypes.c_double, ctypes.c_double, ctypes.c_double]),
    ('dgfs_dg_moments', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
      ctypes.c_void_p]),
    ('dgfs_dg_moments_bi', ctypes.c_int,
     [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int32,
      ctypes.POINTER(ctypes.c_double), ctypes.c_int32, ctypes.c_void_p,
      ctypes.c_void_p]),
    ('dgfs_dg_residual', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
      ctypes.c_int32, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    ('dgfs_penalty_moments', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
      ctypes.c_void_p, ctypes.c_void_p]),
    ('dgfs_penalty_implicit', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
      ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
      ctypes.c_void_p]),
    ('dgfs_penalty_collide', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
      ctypes.c_double, ctypes.c_void_p]),
    ('dgfs_dg_set_limiter', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p]),
    ('dgfs_dg_limit', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    ('dgfs_penalty_moments_n', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
      ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]),
    ('dgfs_penalty_model_relax', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
      ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
      ctypes.c_double, ctypes.c_void_p]),
    ('dgfs_penalty_model_implicit', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
      ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
      ctypes.c_double, ctypes.c_double, ctypes.c_void_p]),
    ('dgfs_penalty_model_collide', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
      ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p]),
    ('dgfs_axnpby', ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_double,
      ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p),
      ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    ('dgfs_vhs_eval_noalloc', ctypes.c_int,
     [ctypes.POINTER(VhsDesc), ctypes.c_void_p, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
      ctypes.c_int32, ctypes.c_void_p]),
]


def lib():
    """Load the library (once) and declare the signatures."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise ImportError(
                f'{LIBPATH} is missing: build it with '
                '`python -m dgfs1d_gpu_b200.build` (nvcc, sm_100a)')
        L = ctypes.CDLL(LIBPATH)
        for name, res, args in _SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc):
    """Raise DgfsError for a non-zero status."""
    if rc != DGFS_OK:
        msg = lib().dgfs_last_error_string()
        raise DgfsError(rc, msg.decode() if msg else '')
    return rc


_deferred = []


def release(destroy, handle):
    """Destroy a native handle (``destroy`` is its dgfs_*_destroy).

    Destroying frees device memory, which a CUDA stream capture does not
    allow: a free issued while a graph is being captured ends that capture
    with an error.  Python may collect an unreachable handle at any moment,
    in the middle of a capture too, so a handle released while this thread's
    current stream is capturing waits in a queue that the next release outside
    a capture empties first."""
    import torch
    if torch.cuda.is_available() and torch.cuda.is_current_stream_capturing():
        _deferred.append((destroy, handle))
        return
    while _deferred:
        d, h = _deferred.pop()
        d(h)
    destroy(handle)


def exported_symbols():
    """Names of every entry point the binding declares."""
    return [s[0] for s in _SIGNATURES]
