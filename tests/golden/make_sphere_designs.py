"""Bundle the symmetric spherical designs into one compressed NumPy file.

The DGFS spherical-quadrature loader (dgfs1D/sphericaldesign/__init__.py:43-105
in the reference) reads Womersley's antipodally symmetric spherical designs,
stored one point per line as ``womersley-ssDDD-mNNNNN.txt`` (DDD = design
degree, NNNNN = point count).  This script converts those published point sets
into ``dgfs1d_gpu_b200/data/womersley_symmetric.npz``, keyed
``ss<DDD>_m<NNNNN>``, so the package can load them on machines where the
reference checkout is absent.

Usage (the directory argument defaults to
``$DGFS_REF/dgfs1D/sphericaldesign/symmetric``)::

    python tests/golden/make_sphere_designs.py [/path/to/sphericaldesign/symmetric]
"""
import os
import re
import sys

import numpy as np


def main(srcdir):
    out = {}
    for name in sorted(os.listdir(srcdir)):
        m = re.match(r'womersley-ss(\d+)-m(\d+)\.txt$', name)
        if not m:
            continue
        pts = np.loadtxt(os.path.join(srcdir, name), dtype=np.float64)
        pts = pts.reshape(-1, 3)
        if len(pts) != int(m.group(2)):
            raise ValueError(f'{name}: expected {m.group(2)} points')
        out['ss%03d_m%05d' % (int(m.group(1)), int(m.group(2)))] = pts
    root = os.path.dirname(os.path.dirname(os.path.dirname(
        os.path.abspath(__file__))))
    dst = os.path.join(root, 'dgfs1d_gpu_b200', 'data',
                       'womersley_symmetric.npz')
    np.savez_compressed(dst, **out)
    print(f'wrote {len(out)} designs to {dst}')


if __name__ == '__main__':
    if len(sys.argv) > 1:
        main(sys.argv[1])
    elif os.environ.get('DGFS_REF'):
        main(os.path.join(os.environ['DGFS_REF'], 'dgfs1D', 'sphericaldesign',
                          'symmetric'))
    else:
        raise SystemExit('give the directory of the symmetric designs, or set '
                         'DGFS_REF to the reference checkout')
