"""The C-ABI library loads and exports every entry point the header declares."""
import os
import re

from dgfs1d_gpu_b200 import _native, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, 'include')):
        if fn.endswith('.h'):
            src = open(os.path.join(ROOT, 'include', fn)).read()
            src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
            names |= set(re.findall(r'\b(dgfs_\w+)\s*\(', src))
    return names


def test_library_exports_header_symbols():
    build.build()
    lib = _native.lib()
    declared = _declared()
    assert declared, 'no declarations found'
    for name in declared:
        assert hasattr(lib, name), f'{name} declared but not exported'
    # the ctypes binding declares every header entry point
    assert declared == set(_native.exported_symbols())


def test_version_string():
    assert b'sm_100a' in _native.lib().dgfs_version()


def test_errors_are_reported_without_gpu():
    import ctypes
    lib = _native.lib()
    h = ctypes.c_void_p()
    rc = lib.dgfs_vhs_create(None, ctypes.byref(h))
    assert rc == -1
    assert b'null' in lib.dgfs_last_error_string()
