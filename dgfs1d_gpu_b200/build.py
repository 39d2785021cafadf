"""Build the in-tree CUDA library ``libdgfs_sm100.so`` for sm_100a.

``python -m dgfs1d_gpu_b200.build`` (or ``build()``) runs nvcc on the single
translation unit ``csrc/dgfs_sm100.cu``; the result sits beside this file so
that it travels with the source tree.  Rebuilds only when a source is newer.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, 'libdgfs_sm100.so')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-shared', '-Xcompiler', '-fPIC']


def sources():
    return (glob.glob(os.path.join(HERE, 'csrc', '*.cu'))
            + glob.glob(os.path.join(HERE, 'csrc', '*.cuh'))
            + glob.glob(os.path.join(ROOT, 'include', '*.h')))


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(s) > t for s in sources())


def build(force=False, verbose=False):
    if not force and not needs_build():
        return OUT
    nvcc = os.environ.get('NVCC', 'nvcc')
    cmd = [nvcc] + ARCH + FLAGS + (['-Xptxas', '-v'] if verbose else []) + [
        '-o', OUT + '.tmp', os.path.join(HERE, 'csrc', 'dgfs_sm100.cu')]
    subprocess.run(cmd, check=True)
    os.replace(OUT + '.tmp', OUT)
    return OUT


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose='-v' in sys.argv))
