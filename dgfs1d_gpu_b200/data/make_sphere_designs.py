"""Bundle the symmetric spherical designs into one compressed NumPy file.

The DGFS spherical-quadrature loader (dgfs1D/sphericaldesign/__init__.py:43-105
in the reference) reads Womersley's antipodally symmetric spherical designs,
stored one point per line as ``womersley-ssDDD-mNNNNN.txt`` (DDD = design
degree, NNNNN = point count).  This script converts those published point sets
into ``womersley_symmetric.npz`` beside it, keyed ``ss<DDD>_m<NNNNN>``, so the
package can load them on machines where the reference checkout is absent.

Usage::

    python make_sphere_designs.py /path/to/dgfs1D/sphericaldesign/symmetric
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
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                       'womersley_symmetric.npz')
    np.savez_compressed(dst, **out)
    print(f'wrote {len(out)} designs to {dst}')


if __name__ == '__main__':
    main(sys.argv[1] if len(sys.argv) > 1 else
         '/root/reference/dgfs1D/sphericaldesign/symmetric')
