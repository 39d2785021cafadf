"""Build recipe: the reference's own CUDA kernels, compiled for the CPU.

Test infrastructure only (see ``oracle/__init__.py``).  The reference's
kernels are Mako templates of CUDA C (dgfs1D/std/kernels/scattering/
vhs-gll.mako, dgfs1D/bi/kernels/scattering/vss.mako, dgfs1D/std/kernels/
std.mako, ...).  This recipe renders a template from the reference checkout
(the directory named by ``$DGFS_REF``, which must be set) with ``oracle.minimako``, prepends a
small prelude that makes the CUDA C compile as C++ (thread indices become
globals set by generated launchers that loop over the grid), and compiles it
with g++ into ``oracle/_ref/`` (git-ignored).  Nothing of the reference is
copied into the repository; only the rendered, compiled object is produced,
and only into ``oracle/_ref``.

Used by ``tests/golden/make_golden.py`` to produce golden vectors from the
reference's own arithmetic (cuFFT, a closed library, is replaced by pocketfft
there, exactly as in the oracle).
"""
import ctypes
import hashlib
import os
import re
import subprocess

import numpy as np

from .minimako import render

REF = os.environ.get('DGFS_REF')
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), '_ref')

PRELUDE = r'''
#include <cmath>
#include <cstdint>
struct dgfs_dim3 { unsigned x, y, z; };
static dgfs_dim3 blockIdx, threadIdx, blockDim, gridDim;
#define __global__ static
#define __device__
#define __host__
#define __shared__ static
#define __syncthreads()
#define __restrict__
typedef struct { double x, y; } cufftDoubleComplex;
typedef struct { float x, y; } cufftComplex;
using std::sin; using std::cos; using std::pow; using std::sqrt; using std::fabs;
using std::exp;
// CUDA's overloaded min/max for double and int operands
static inline double min(double a, double b) { return a < b ? a : b; }
static inline double max(double a, double b) { return a > b ? a : b; }
static inline int min(int a, int b) { return a < b ? a : b; }
static inline int max(int a, int b) { return a > b ? a : b; }
'''


def template_path(rel):
    if not REF:
        raise RuntimeError('set DGFS_REF to the reference checkout (the '
                           'directory that holds dgfs1D/)')
    return os.path.join(REF, rel)


def render_template(rel, **kw):
    with open(template_path(rel)) as fh:
        src = fh.read()
    return render(src, **kw)


_SIG = re.compile(r'__global__\s+void\s+(\w+)\s*\((.*?)\)\s*\{', re.S)


def _params(sig):
    out = []
    for p in sig.split(','):
        p = re.sub(r'//[^\n]*', '', p).strip()
        if not p:
            continue
        name = re.findall(r'(\w+)\s*$', p)[0]
        ctype = p[:p.rfind(name)].strip()
        out.append((ctype, name))
    return out


def _ctypes_of(ctype):
    if '*' in ctype:
        return ctypes.c_void_p
    base = ctype.replace('const', '').strip()
    if base in ('int',):
        return ctypes.c_int
    if base in ('unsigned int', 'unsigned'):
        return ctypes.c_uint
    if base in ('double', 'scalar'):
        return ctypes.c_double
    if base == 'float':
        return ctypes.c_float
    raise ValueError(f'unsupported kernel parameter type {ctype!r}')


class RefModule:
    """A rendered reference template compiled for the CPU.

    ``launch(name, grid, block, *args)`` runs the kernel over the 1-D grid;
    numpy arrays are passed by pointer, scalars by value.
    """

    def __init__(self, src, scalar='double', tag='ref'):
        kernels = _SIG.findall(src)
        self.sigs = {k: _params(a) for k, a in kernels}
        launchers = []
        for name, params in self.sigs.items():
            decl = ', '.join(f'{t} a{i}' for i, (t, _) in enumerate(params))
            call = ', '.join(f'a{i}' for i in range(len(params)))
            launchers.append(
                f'extern "C" void launch_{name}(unsigned grid, unsigned block'
                f'{", " if decl else ""}{decl}) {{\n'
                f'  blockDim.x = block; blockDim.y = blockDim.z = 1;\n'
                f'  gridDim.x = grid; gridDim.y = gridDim.z = 1;\n'
                f'  for (unsigned b = 0; b < grid; ++b)\n'
                f'    for (unsigned t = 0; t < block; ++t) {{\n'
                f'      blockIdx.x = b; threadIdx.x = t;\n'
                f'      {name}({call});\n'
                f'    }}\n}}\n')
        full = PRELUDE + src.replace('#include <cufft.h>', '') + '\n' + \
            '\n'.join(launchers)
        # scalar typedefs used by templates that rely on #define scalar
        os.makedirs(OUT, exist_ok=True)
        h = hashlib.sha1(full.encode()).hexdigest()[:16]
        so = os.path.join(OUT, f'{tag}-{h}.so')
        if not os.path.exists(so):
            cpp = so[:-3] + '.cpp'
            with open(cpp, 'w') as fh:
                fh.write(full)
            subprocess.run(['g++', '-O1', '-fno-fast-math', '-ffp-contract=off',
                            '-shared', '-fPIC', '-o', so, cpp], check=True)
        self.lib = ctypes.CDLL(so)
        for name, params in self.sigs.items():
            fn = getattr(self.lib, 'launch_' + name)
            fn.restype = None
            fn.argtypes = [ctypes.c_uint, ctypes.c_uint] + \
                [_ctypes_of(t) for t, _ in params]

    def launch(self, name, grid, block, *args):
        conv = []
        for a in args:
            if isinstance(a, np.ndarray):
                if not a.flags['C_CONTIGUOUS']:
                    raise ValueError('arrays must be contiguous')
                conv.append(a.ctypes.data)
            else:
                conv.append(a)
        getattr(self.lib, 'launch_' + name)(grid, block, *conv)


def grid_for(n, block):
    return (n + block - 1) // block
